// Panel factorization inside one thread-block cluster, with the per-column
// pivot exchange done by pushes into the peers' shared memory.
//
// Same arithmetic as k_panel / k_panel_cluster (the reference's panel:
// src/matrix_operation/cpu/native/lu_decomposition_native.cpp:158-232):
// per column the first largest |a| in row order wins (a NaN never displaces,
// a NaN on the diagonal is never displaced), the row swap covers the panel's
// columns, the multipliers are a * (1/d) when |d| >= the smallest normal
// value (else a / d), and every element below is updated with one fused
// multiply-add per column in column order.  Factors and pivots are therefore
// bit-identical to the other panel kernels.
//
// Exchange, per column c (one CTA barrier and one one-way push per column):
//   * warp 0 of every CTA reduces its warps' candidates and stores the
//     record {key, row, the candidate row's W values} into slot [c % 2][rank]
//     of EVERY CTA of the cluster (st.async into distributed shared memory,
//     completing on the receiver's mbarrier for that slot parity); warp 1 of
//     the CTA that holds row c stores row c the same way;
//   * every thread waits on its own CTA's mbarrier (all records and row c
//     have landed), reduces the CL records itself and so knows the pivot
//     row p and its values without reading another CTA's memory;
//   * the owner of row c writes the pivot row there, the owner of row p
//     takes row c while it updates row p, and all rows below c are updated,
//     their next-column candidates reduced per warp; one __syncthreads.
// Each pushing warp stores into its own CTA last (after a __syncwarp), so no
// thread passes the wait before those warps have read everything they push:
// the update that follows cannot race with the reads of the push.  A slot of parity q is
// rewritten two columns later, after every CTA has passed the barrier that
// ends the column in between, so it is never overwritten while being read.
// Every wait is bounded (2 s): on expiry the kernel records
// DEV_WAIT_TIMEOUT, and all CTAs meet at a final cluster barrier before any
// of them exits (no store can target an exited CTA).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cfloat>
#include <climits>

#include "lu_kernels.cuh"

namespace b200la
{

constexpr int    kPushThreads  = 256;
constexpr int    kPushWarps    = kPushThreads / 32;
constexpr int    kPushMaxCl    = 16;
// dynamic shared memory: sm_100's 227 KB per CTA less 2 KB for the static
// arrays of build_perm_list
constexpr size_t kPushSmemMax  = 227 * 1024 - 2048;

// Shared-memory layout of k_panel_push for panel width W (bytes).
template <typename T, int W> struct PushLayout
{
    static constexpr int    ldl        = W + 16 / (int)sizeof(T);  // slice row stride (elements)
    static constexpr int    rec_bytes  = 16 + W * (int)sizeof(T);  // {key, row, pad} + the row
    static constexpr int    rec_chunks = rec_bytes / 16;
    static constexpr int    row_chunks = W * (int)sizeof(T) / 16;
    static constexpr size_t slots      = 0;                                            // [2][kPushMaxCl] records
    static constexpr size_t crow       = slots + (size_t)2 * kPushMaxCl * rec_bytes;  // [2][W]: row c
    static constexpr size_t bars       = crow + (size_t)2 * W * sizeof(T);            // 2 mbarriers
    static constexpr size_t red_key    = bars + 16;                                   // [kPushWarps] double
    static constexpr size_t red_row    = red_key + 8 * kPushWarps;                    // [kPushWarps] int
    static constexpr size_t piv        = red_row + 4 * kPushWarps;                    // [W] int
    static constexpr size_t head       = (piv + 4 * W + 15) / 16 * 16;
    static constexpr size_t row_bytes  = (size_t)ldl * sizeof(T);
    static_assert(rec_bytes % 16 == 0 && (W * sizeof(T)) % 16 == 0, "16-byte pushes");
};

template <typename T, int W> constexpr size_t push_smem_bytes(int rows_per_cta)
{
    return PushLayout<T, W>::head + (size_t)rows_per_cta * PushLayout<T, W>::row_bytes;
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
// 16 bytes into another CTA's shared memory (or this CTA's), completing as
// 16 transaction bytes on that CTA's mbarrier at the same offset as ours.
__device__ __forceinline__ void push16(uint32_t remote_addr, uint4 v, uint32_t remote_bar)
{
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(
                     remote_addr),
        "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "r"(remote_bar)
        : "memory");
}
__device__ __forceinline__ void fence_mbarrier_init_cluster()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Copy the panel slice (nloc rows of w values at A[r0.., k..], row stride n)
// into shared memory (row stride LDL) or back; 16-byte vectors when the
// rows allow it, 8 loads of a thread in flight before its stores.
template <typename T, int LDL, bool TO_SMEM>
__device__ __forceinline__ void push_slice_copy(T* loc, T* A, int n, int r0, int k, int nloc, int w)
{
    using VT          = typename Vec16<T>::type;
    constexpr int V   = 16 / (int)sizeof(T);
    constexpr int B   = 8;
    const bool    vec = (w % V) == 0 && (n % V) == 0 && (k % V) == 0 && (reinterpret_cast<uintptr_t>(A) & 15) == 0;
    if (vec)
    {
        const int cpr   = w / V;
        const int total = nloc * cpr;
        for (int e0 = threadIdx.x; e0 < total; e0 += kPushThreads * B)
        {
            VT v[B];
#pragma unroll
            for (int t = 0; t < B; ++t)
            {
                const int e = e0 + t * kPushThreads;
                if (e < total)
                {
                    const int r = e / cpr, c = (e - r * cpr) * V;
                    v[t]        = TO_SMEM ? *reinterpret_cast<const VT*>(A + (size_t)(r0 + r) * n + k + c)
                                          : *reinterpret_cast<const VT*>(loc + (size_t)r * LDL + c);
                }
            }
#pragma unroll
            for (int t = 0; t < B; ++t)
            {
                const int e = e0 + t * kPushThreads;
                if (e < total)
                {
                    const int r = e / cpr, c = (e - r * cpr) * V;
                    if (TO_SMEM)
                        *reinterpret_cast<VT*>(loc + (size_t)r * LDL + c) = v[t];
                    else
                        *reinterpret_cast<VT*>(A + (size_t)(r0 + r) * n + k + c) = v[t];
                }
            }
        }
        return;
    }
    const int total = nloc * w;
    for (int e = threadIdx.x; e < total; e += kPushThreads)
    {
        const int r = e / w, c = e - r * w;
        if (TO_SMEM)
            loc[(size_t)r * LDL + c] = A[(size_t)(r0 + r) * n + k + c];
        else
            A[(size_t)(r0 + r) * n + k + c] = loc[(size_t)r * LDL + c];
    }
}

template <typename T, int W>
__global__ void __launch_bounds__(kPushThreads, 1) k_panel_push(T* __restrict__ A, int n, int k, int w,
    int rows_per_cta, int64_t* __restrict__ pivot, PermList* __restrict__ perm, DeviceStatus* __restrict__ st)
{
    using L = PushLayout<T, W>;
    using VT          = typename Vec16<T>::type;
    constexpr int V   = 16 / (int)sizeof(T);
    constexpr int LDL = L::ldl;
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char* slots   = smem + L::slots;
    T*             crow    = reinterpret_cast<T*>(smem + L::crow);
    uint64_t*      bar     = reinterpret_cast<uint64_t*>(smem + L::bars);
    double*        red_key = reinterpret_cast<double*>(smem + L::red_key);
    int*           red_row = reinterpret_cast<int*>(smem + L::red_row);
    int*           piv_loc = reinterpret_cast<int*>(smem + L::piv);
    T*             loc     = reinterpret_cast<T*>(smem + L::head);

    const int      tid  = threadIdx.x;
    const int      lane = tid & 31;
    const int      warp = tid >> 5;
    const uint32_t CL   = cluster_size();
    const uint32_t b    = cluster_rank();
    const int      r0   = k + (int)b * rows_per_cta;
    const int      nloc = max(0, min(n, r0 + rows_per_cta) - r0);
    const uint32_t tx   = CL * (uint32_t)L::rec_bytes + (uint32_t)(W * sizeof(T));

    if (tid == 0)
    {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbarrier_init_cluster();
        mbar_expect_tx(&bar[0], tx);  // column 0
        if (w > 1)
        {
            mbar_expect_tx(&bar[1], tx);  // column 1
        }
    }
    push_slice_copy<T, LDL, true>(loc, A, n, r0, k, nloc, w);
    __syncthreads();

    // candidate of column k
    double ck = -2.0;
    int    cr = INT_MAX;
    for (int r = max(0, k - r0) + tid; r < nloc; r += kPushThreads)
    {
        const double key = pivot_key(loc[(size_t)r * LDL], r0 + r, k);
        if (better(key, r0 + r, ck, cr))
        {
            ck = key;
            cr = r0 + r;
        }
    }
    warp_best(ck, cr);
    if (lane == 0)
    {
        red_key[warp] = ck;
        red_row[warp] = cr;
    }
    cluster_barrier();  // every CTA's mbarriers are initialized; red_* visible to all threads

    int64_t first_zero = -1;
    bool    aborted    = false;
    for (int jj = 0; jj < w; ++jj)
    {
        const int      c      = k + jj;
        const int      par    = jj & 1;
        const uint32_t parity = (uint32_t)(jj >> 1) & 1u;
        const uint32_t rank_c = (uint32_t)((c - k) / rows_per_cta);
        const uint32_t bar_l  = smem_u32(&bar[par]);
        // ---- push: warp 0 this CTA's candidate record, warp 1 (owner of row c) row c
        if (warp == 0)
        {
            double bk = red_key[0];
            int    br = red_row[0];
#pragma unroll
            for (int q = 1; q < kPushWarps; ++q)
            {
                if (better(red_key[q], red_row[q], bk, br))
                {
                    bk = red_key[q];
                    br = red_row[q];
                }
            }
            const unsigned char* src = br != INT_MAX ? reinterpret_cast<const unsigned char*>(loc + (size_t)(br - r0) * LDL)
                                                     : nullptr;
            const uint32_t rec_l = smem_u32(slots + ((size_t)par * kPushMaxCl + b) * L::rec_bytes);
            const uint64_t kb    = (uint64_t)__double_as_longlong(bk);
            auto chunk = [&](int ch) {
                if (ch == 0)
                {
                    return make_uint4((uint32_t)kb, (uint32_t)(kb >> 32), (uint32_t)br, 0u);
                }
                return src != nullptr ? *reinterpret_cast<const uint4*>(src + (ch - 1) * 16)
                                      : make_uint4(0u, 0u, 0u, 0u);
            };
            // the other CTAs first (b+1, b+2, ...), then, once every lane is
            // done with them, this CTA
            for (int i = lane; i < ((int)CL - 1) * L::rec_chunks; i += 32)
            {
                const int      qi   = i / L::rec_chunks;
                const int      ch   = i - qi * L::rec_chunks;
                const uint32_t peer = (b + 1 + (uint32_t)qi) % CL;
                push16(map_to_rank(rec_l + ch * 16, peer), chunk(ch), map_to_rank(bar_l, peer));
            }
            __syncwarp();
            for (int ch = lane; ch < L::rec_chunks; ch += 32)
            {
                push16(map_to_rank(rec_l + ch * 16, b), chunk(ch), map_to_rank(bar_l, b));
            }
        }
        else if (warp == 1 && b == rank_c)
        {
            const unsigned char* src    = reinterpret_cast<const unsigned char*>(loc + (size_t)(c - r0) * LDL);
            const uint32_t       crow_l = smem_u32(crow + (size_t)par * W);
            for (int i = lane; i < ((int)CL - 1) * L::row_chunks; i += 32)
            {
                const int      qi   = i / L::row_chunks;
                const int      ch   = i - qi * L::row_chunks;
                const uint32_t peer = (b + 1 + (uint32_t)qi) % CL;
                push16(map_to_rank(crow_l + ch * 16, peer), *reinterpret_cast<const uint4*>(src + ch * 16),
                    map_to_rank(bar_l, peer));
            }
            __syncwarp();
            for (int ch = lane; ch < L::row_chunks; ch += 32)
            {
                push16(map_to_rank(crow_l + ch * 16, b), *reinterpret_cast<const uint4*>(src + ch * 16),
                    map_to_rank(bar_l, b));
            }
        }
        // ---- wait for every record and row c
        const bool ok = mbar_wait(&bar[par], parity);
        double     nk = -2.0;
        int        nr = INT_MAX;
        if (ok)
        {
            if (tid == 0 && jj + 2 < w)
            {
                mbar_expect_tx(&bar[par], tx);  // arm the slot parity for column jj + 2
            }
            // the pivot: every thread reduces the CL records itself
            double   pk     = -3.0;
            int      p      = INT_MAX;
            uint32_t rank_p = 0;
            for (uint32_t q = 0; q < CL; ++q)
            {
                const unsigned char* rec = slots + ((size_t)par * kPushMaxCl + q) * L::rec_bytes;
                const double         kq  = *reinterpret_cast<const double*>(rec);
                const int            rq  = *reinterpret_cast<const int*>(rec + 8);
                if (better(kq, rq, pk, p))
                {
                    pk     = kq;
                    p      = rq;
                    rank_p = q;
                }
            }
            const T* urow = reinterpret_cast<const T*>(slots + ((size_t)par * kPushMaxCl + rank_p) * L::rec_bytes + 16);
            const T* crw  = crow + (size_t)par * W;
            if (tid == 0)
            {
                piv_loc[jj] = p;
                if (b == 0)
                {
                    pivot[c] = (int64_t)p + 1;
                }
            }
            const T d = urow[jj];
            if (d == T(0) && first_zero < 0)
            {
                first_zero = c;
            }
            // row c <- the pivot row (its owner; no other thread touches row c
            // in this column)
            if (b == rank_c && p != c)
            {
                for (int cc = tid; cc < w; cc += kPushThreads)
                {
                    loc[(size_t)(c - r0) * LDL + cc] = urow[cc];
                }
            }
            const bool own_p     = p != c && p >= r0 && p < r0 + nloc;
            const bool zero      = d == T(0);
            const bool use_recip = fabs(d) >= Limits<T>::min_normal();
            const T    recip     = use_recip ? (T)(T(1) / d) : T(1);
            const bool has_next  = jj + 1 < w;
            for (int r = max(0, c + 1 - r0) + tid; r < nloc; r += kPushThreads)
            {
                T*         row     = loc + (size_t)r * LDL;
                const bool swapped = own_p && r0 + r == p;
                const T*   srow    = swapped ? crw : row;
                if (swapped)
                {
                    for (int cc = 0; cc < jj; ++cc)
                    {
                        row[cc] = crw[cc];  // row c's multipliers travel with it
                    }
                }
                if (!zero)
                {
                    const T x = srow[jj];
                    const T l = use_recip ? x * recip : x / d;
                    row[jj]   = l;
                    int cc    = jj + 1;
                    for (; cc < w && (cc % V) != 0; ++cc)
                    {
                        row[cc] = fma(-l, urow[cc], srow[cc]);
                    }
                    for (; cc + V <= w; cc += V)
                    {
                        const VT sv = *reinterpret_cast<const VT*>(srow + cc);
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
                    for (; cc < w; ++cc)
                    {
                        row[cc] = fma(-l, urow[cc], srow[cc]);
                    }
                }
                else if (swapped)
                {
                    for (int cc = jj; cc < w; ++cc)
                    {
                        row[cc] = crw[cc];
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
        warp_best(nk, nr);
        if (lane == 0)
        {
            red_key[warp] = nk;
            red_row[warp] = nr;
        }
        if (__syncthreads_or(ok ? 0 : 1))
        {
            if (tid == 0)
            {
                raise_error(st, DEV_WAIT_TIMEOUT, 4);
            }
            aborted = true;
            break;
        }
    }
    cluster_barrier();  // no CTA exits while a peer may still store into it

    push_slice_copy<T, LDL, false>(loc, A, n, r0, k, nloc, w);
    if (b == 0 && !aborted)
    {
        if (tid == 0 && first_zero >= 0 && st->first_zero < 0)
        {
            st->first_zero = first_zero;
        }
        if (warp == 0)
        {
            build_perm_list(piv_loc, k, w, perm, lane);
        }
    }
}

// The floor of k_panel_push's per-column exchange: the same cluster, the
// same record and row-c pushes (self last), the same bounded wait, pivot
// reduction over the CL records and end-of-column barrier, but no panel
// slice, no update and no candidate search.  Thread 0 of rank 0 writes the
// elapsed %globaltimer nanoseconds of `columns` columns to *ns.
template <typename T, int W>
__global__ void __launch_bounds__(kPushThreads, 1) k_panel_exchange_floor(int columns,
    unsigned long long* __restrict__ ns, DeviceStatus* __restrict__ st)
{
    using L = PushLayout<T, W>;
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char* slots   = smem + L::slots;
    T*             crow    = reinterpret_cast<T*>(smem + L::crow);
    uint64_t*      bar     = reinterpret_cast<uint64_t*>(smem + L::bars);
    double*        red_key = reinterpret_cast<double*>(smem + L::red_key);
    int*           red_row = reinterpret_cast<int*>(smem + L::red_row);
    const int      tid     = threadIdx.x;
    const int      lane    = tid & 31;
    const int      warp    = tid >> 5;
    const uint32_t CL      = cluster_size();
    const uint32_t b       = cluster_rank();
    const uint32_t tx      = CL * (uint32_t)L::rec_bytes + (uint32_t)(W * sizeof(T));
    if (tid == 0)
    {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbarrier_init_cluster();
        mbar_expect_tx(&bar[0], tx);
        mbar_expect_tx(&bar[1], tx);
    }
    if (lane == 0)
    {
        red_key[warp] = (double)(warp * 7 % 5);
        red_row[warp] = warp + (int)b * 100;
    }
    cluster_barrier();
    const uint64_t t0 = global_ns();
    for (int jj = 0; jj < columns; ++jj)
    {
        const int      par    = jj & 1;
        const uint32_t parity = (uint32_t)(jj >> 1) & 1u;
        const uint32_t bar_l  = smem_u32(&bar[par]);
        if (warp == 0)
        {
            double bk = red_key[0];
            int    br = red_row[0];
            for (int q = 1; q < kPushWarps; ++q)
            {
                if (better(red_key[q], red_row[q], bk, br))
                {
                    bk = red_key[q];
                    br = red_row[q];
                }
            }
            const uint32_t rec_l = smem_u32(slots + ((size_t)par * kPushMaxCl + b) * L::rec_bytes);
            const uint64_t kb    = (uint64_t)__double_as_longlong(bk);
            const uint4    hdr   = make_uint4((uint32_t)kb, (uint32_t)(kb >> 32), (uint32_t)br, 0u);
            const uint4    val   = make_uint4((uint32_t)jj, 0u, 0u, 0u);
            for (int i = lane; i < ((int)CL - 1) * L::rec_chunks; i += 32)
            {
                const int      qi   = i / L::rec_chunks;
                const int      ch   = i - qi * L::rec_chunks;
                const uint32_t peer = (b + 1 + (uint32_t)qi) % CL;
                push16(map_to_rank(rec_l + ch * 16, peer), ch == 0 ? hdr : val, map_to_rank(bar_l, peer));
            }
            __syncwarp();
            for (int ch = lane; ch < L::rec_chunks; ch += 32)
            {
                push16(map_to_rank(rec_l + ch * 16, b), ch == 0 ? hdr : val, map_to_rank(bar_l, b));
            }
        }
        else if (warp == 1 && b == (uint32_t)jj % CL)
        {
            const uint32_t crow_l = smem_u32(crow + (size_t)par * W);
            const uint4    val    = make_uint4((uint32_t)jj, 1u, 0u, 0u);
            for (int i = lane; i < ((int)CL - 1) * L::row_chunks; i += 32)
            {
                const int      qi   = i / L::row_chunks;
                const int      ch   = i - qi * L::row_chunks;
                const uint32_t peer = (b + 1 + (uint32_t)qi) % CL;
                push16(map_to_rank(crow_l + ch * 16, peer), val, map_to_rank(bar_l, peer));
            }
            __syncwarp();
            for (int ch = lane; ch < L::row_chunks; ch += 32)
            {
                push16(map_to_rank(crow_l + ch * 16, b), val, map_to_rank(bar_l, b));
            }
        }
        const bool ok = mbar_wait(&bar[par], parity);
        double     nk = -2.0;
        int        nr = INT_MAX;
        if (ok)
        {
            if (tid == 0 && jj + 2 < columns)
            {
                mbar_expect_tx(&bar[par], tx);
            }
            for (uint32_t q = 0; q < CL; ++q)
            {
                const unsigned char* rec = slots + ((size_t)par * kPushMaxCl + q) * L::rec_bytes;
                const double         kq  = *reinterpret_cast<const double*>(rec);
                const int            rq  = *reinterpret_cast<const int*>(rec + 8);
                if (better(kq, rq, nk, nr))
                {
                    nk = kq;
                    nr = rq;
                }
            }
        }
        warp_best(nk, nr);
        if (lane == 0)
        {
            red_key[warp] = nk;
            red_row[warp] = nr - (int)b;
        }
        if (__syncthreads_or(ok ? 0 : 1))
        {
            if (tid == 0)
            {
                raise_error(st, DEV_WAIT_TIMEOUT, 5);
            }
            break;
        }
    }
    const uint64_t t1 = global_ns();
    cluster_barrier();
    if (b == 0 && tid == 0)
    {
        *ns = t1 - t0;
    }
}

}  // namespace b200la
