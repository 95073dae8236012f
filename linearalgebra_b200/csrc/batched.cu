// Batched solver for many independent dense systems of uneven order
// (1 <= n <= 512), in ONE persistent kernel launch.
//
// A CTA of 256 threads works in groups of G threads (G = 256, 128 or 64),
// one system per group at a time: the CTA's first group takes the next system
// from an atomic queue (the caller orders the systems largest first), reads
// the group size and panel width that the autotuner chose for its order
// bucket, and every other group takes one more system; each group then solves
// its system with its own named barrier, and the CTA meets again.  Per
// system:
//   * A (FP64, global) is copied into the group's factor scratch in the
//     factorization type T (float: FP32 factors + FP64 refinement; double:
//     plain FP64 LU), row stride padded to 16 bytes, with ||A||_inf on the
//     way;
//   * blocked right-looking LU with partial pivoting, panel width NB.  Rows
//     never move in the scratch: a logical-to-physical row map takes every
//     interchange, so a panel's interchanges cost one map update instead of a
//     gather and scatter of whole rows, and the map is the solve's row
//     permutation at the end;
//       - the panel (all remaining rows x NB columns) is factored in
//         registers (RPT rows per thread, rows staying in their thread with
//         their current position in a register, when the rows fit) or in
//         shared memory: per column a pivot search (integer keys,
//         redux.sync), the pivot row posted through shared memory, and the
//         rank-1 update;
//       - U12 = L11^-1 A12, one thread per column;
//       - A22 -= L21 U12 with 8 x 8 (FP32) or 4 x 8 (FP64) register tiles per
//         thread: the tile of A22 is loaded (16-byte vectors) before the
//         product, L21 (transposed) and U12 come from shared memory in
//         16-byte vectors without bank conflicts;
//   * the solve applies the factors in FP64: 32-row blocks in solve order;
//     for each block the products with the solved values are dot products
//     over whole factor rows read by G / 32 threads per row (16-byte
//     vectors), the diagonal block is staged in shared memory and solved in
//     one warp's registers (rows by lane, substitution with shuffles); then
//     FP64 refinement r = b - A x, d = U^-1 L^-1 P r, x += d until the
//     normwise backward error ||r|| / (||A|| ||x|| + ||b||) <= tol, the
//     refinement stalls (less than a factor 2 gained per correction after
//     the first) or max_iter corrections.
// With FP32 factors a second launch with FP64 factors takes only the
// systems whose refinement did not converge (ill-conditioned ones); it
// skips every other system at the cost of one queue step.
// Per-system outputs: status (corrections used, 1000 + corrections after the
// FP64 pass, -(info) for an exactly singular U, -1000000 if not converged)
// and the final backward error.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>

#include "common.cuh"

// Phase hook: B200LA_BPHASE(i) marks the end of phase i of a system's solve
// (nothing by default; a timing harness may define it before including this
// file).
#ifndef B200LA_BPHASE
#define B200LA_BPHASE(i) \
    do                   \
    {                    \
    } while (0)
#endif

namespace b200la
{
namespace
{
constexpr int kBT       = 256;  // threads per CTA
constexpr int kBMaxN    = 512;
constexpr int kBBuckets = 8;    // order buckets of 64
constexpr int kBSolveNB = 32;   // rows per block of the triangular solves
constexpr int kBDgLd    = kBSolveNB + 1;
// factor scratch: one slot of kBScratch bytes per CTA (split between the
// CTA's groups), at most kBMaxCTAs slots
constexpr size_t kBScratch = (size_t)kBMaxN * kBMaxN * sizeof(double);
constexpr int    kBMaxCTAs = 192;
// status of a system whose refinement stalled or ran out of corrections; the
// FP64 pass picks these up.  Systems finished by that pass get 1000 + k.
constexpr int32_t kNotConverged = -1000000;
constexpr int32_t kEscalated    = 1000;

template <typename T> struct BatchTraits;
template <> struct BatchTraits<float>
{
    static constexpr int kMaxNB = 32;
    static constexpr int kMinNB = 16;
    static constexpr int TM     = 8;  // rows of a thread's update tile (8 x 8)
};
template <> struct BatchTraits<double>
{
    static constexpr int kMaxNB = 16;
    static constexpr int kMinNB = 8;
    static constexpr int TM     = 4;  // 4 x 8
};

// A bucket's table entry: bits 0-7 the panel width NB, bits 8-15 the
// threads per system / 32 (0: the whole CTA).
__host__ __device__ inline int entry_nb(int e) { return e & 0xff; }
__host__ __device__ inline int entry_g(int e)
{
    const int g = ((e >> 8) & 0xff) * 32;
    return g == 64 || g == 128 ? g : kBT;
}
// The panel widths the kernel is built for: kMaxNB or kMinNB.
template <typename T> __host__ __device__ inline bool nb_supported(int nb)
{
    return nb == BatchTraits<T>::kMaxNB || nb == BatchTraits<T>::kMinNB;
}

__host__ __device__ inline int group_np(int n) { return (n + 7) / 8 * 8 + 8; }
// Row stride of the factor scratch: n rounded up to 16 bytes.
template <typename T> __host__ __device__ inline int bat_ld(int n)
{
    constexpr int v = 16 / (int)sizeof(T);
    return (n + v - 1) / v * v;
}

// Rows per thread of the register panel for order n and G threads: 2 or 4
// (4 only while RPT x NB stays within 64 FP32 / 32 FP64 values), 0 if the
// panel is factored in shared memory.
template <typename T> __host__ __device__ inline int panel_rpt(int n, int nb, int G)
{
    if (n <= 2 * G)
        return 2;
    if (n <= 4 * G && 4 * nb * (int)sizeof(T) <= 256)
        return 4;
    return 0;
}

// Shared-memory slice of one group of G threads solving a system of order n
// with panel width nb (the same function sizes and carves).
struct GroupSmem
{
    size_t P, LT, U, y, r, x, dg, dpart, sigma, list, rowp, red, end;
};
template <typename T> __host__ __device__ inline GroupSmem group_layout(int n, int nb, int G)
{
    auto up = [](size_t v) { return (v + 15) / 16 * 16; };
    const int np = group_np(n);      // padded rows of LT and U (the update tiles read past n)
    const int nv = n > 16 ? n : 16;  // FP64 vectors (also the group's reductions: 2 per warp)
    // the register panel keeps only L11 in P, the shared-memory panel all rows
    const int prow = panel_rpt<T>(n, nb, G) != 0 ? nb : n;
    GroupSmem g;
    g.P     = 0;                                              // T[prow][nb + 1]: the panel
    g.LT    = up(g.P + sizeof(T) * (size_t)prow * (nb + 1));  // T[nb][np]: L21 transposed
    g.U     = up(g.LT + sizeof(T) * (size_t)nb * np);      // T[nb][np]: U12
    g.y     = up(g.U + sizeof(T) * (size_t)nb * np);       // double[nv]
    g.r     = up(g.y + sizeof(double) * nv);               // double[nv]
    g.x     = up(g.r + sizeof(double) * nv);               // double[nv]
    g.dg    = up(g.x + sizeof(double) * nv);               // T[32][33]: diagonal block / posted rows
    g.dpart = up(g.dg + sizeof(T) * kBSolveNB * kBDgLd);   // double[32]: the block's products
    g.sigma = up(g.dpart + sizeof(double) * kBSolveNB);    // int[n]: the panel's row order
    g.list  = up(g.sigma + sizeof(int) * n);               // int[4 nb]: moved rows, their old map
    g.rowp  = up(g.list + sizeof(int) * 4 * nb);           // int[n]: logical -> physical row
    g.red   = up(g.rowp + sizeof(int) * n);                // 8 x (u64 key, int row) + flags
    g.end   = up(g.red + 8 * 8 + 8 * 4 + 64);
    return g;
}

constexpr size_t kBatchedSmem = 227 * 1024 - 1024;  // dynamic shared memory per CTA

__host__ __device__ inline size_t group_smem_bytes(int G) { return kBatchedSmem / (kBT / G) / 16 * 16; }
__host__ __device__ inline size_t group_scratch_bytes(int G) { return kBScratch / (kBT / G); }

// Whether a system of order n fits a group of G threads with panel width nb.
template <typename T> __host__ __device__ inline bool group_fits(int n, int nb, int G)
{
    return group_layout<T>(n, nb, G).end <= group_smem_bytes(G) &&
           (size_t)n * bat_ld<T>(n) * sizeof(T) <= group_scratch_bytes(G);
}

__device__ __forceinline__ void group_sync(int id, int threads)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

template <typename T> struct BKey;
template <> struct BKey<float>
{
    using type = uint32_t;
};
template <> struct BKey<double>
{
    using type = unsigned long long;
};
// Pivot-search key (larger wins, ties to the lower row): |v|'s bits + 2; 1
// for a NaN below the diagonal, the maximum for one on it, 0 for none.
template <typename T> __device__ __forceinline__ typename BKey<T>::type bkey(T v, bool diag)
{
    using K = typename BKey<T>::type;
    if (v != v)
        return diag ? ~K(0) : K(1);
    if constexpr (sizeof(T) == 4)
        return (K)__float_as_uint(fabsf(v)) + K(2);
    else
        return (K)__double_as_longlong(fabs(v)) + K(2);
}
template <typename K> __device__ __forceinline__ void bwarp_best(K& key, int& row)
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

// 16-byte vector <-> elements
template <typename T> __device__ __forceinline__ void vload(const T* p, T* e)
{
    if constexpr (sizeof(T) == 4)
    {
        const float4 v = *reinterpret_cast<const float4*>(p);
        e[0] = v.x, e[1] = v.y, e[2] = v.z, e[3] = v.w;
    }
    else
    {
        const double2 v = *reinterpret_cast<const double2*>(p);
        e[0] = v.x, e[1] = v.y;
    }
}
template <typename T> __device__ __forceinline__ void vstore(T* p, const T* e)
{
    if constexpr (sizeof(T) == 4)
    {
        *reinterpret_cast<float4*>(p) = make_float4(e[0], e[1], e[2], e[3]);
    }
    else
    {
        *reinterpret_cast<double2*>(p) = make_double2(e[0], e[1]);
    }
}

// One group's state for one system.
template <typename T> struct Sys
{
    int      n, nb, G, gt, bar;  // order, panel width, threads, this thread's index, barrier id
    int      ld;                 // row stride of f
    T*       f;                  // factor scratch (global), n rows of stride ld, rows in physical order
    T*       P;                  // [n][nb + 1]
    T*       LT;                 // [nb][np]
    T*       U;                  // [nb][np]
    int      np;
    double * y, *r, *x;
    T*       dg;     // [32][33]
    double*  dpart;  // [32]
    int *    sigma, *list, *rowp;
    unsigned long long* red_key;
    int*                red_row;
    int*                flags;  // [0] first zero pivot (-1 none), [1] list count

    __device__ void sync() const { group_sync(bar, G); }
    __device__ T*   row(int logical) const { return f + (size_t)rowp[logical] * ld; }
};

// y <- T^-1 y for the unit-lower (upper = false) or upper triangle of the
// factor (FP64 arithmetic).  32-row blocks in solve order.  Per block: the
// block's rows times the values already solved, G / 32 threads per row, each
// on 16-byte vectors of the row, summed with shuffles; then warp 0 holds the
// diagonal block (staged in shared memory) in registers, row b0 + lane, and
// substitutes with shuffles (the upper triangle's divisions as products with
// reciprocals each lane takes beforehand).  A block's first kTrPre vectors
// per thread and its diagonal block are loaded while the block before it is
// substituted: the loads do not depend on the values being solved.
constexpr int kTrPre = 16;
template <typename T> __device__ void bat_trsv(const Sys<T>& s, bool upper)
{
    constexpr int VN   = 16 / (int)sizeof(T);
    constexpr int DV   = kBSolveNB / VN / 2;  // diagonal-block vectors per thread, at most (2+ threads per row)
    const int     lane = s.gt & 31, warp = s.gt >> 5;
    const int     n    = s.n;
    const int     nblk = (n + kBSolveNB - 1) / kBSolveNB;
    const int     tpr  = s.G >> 5;  // threads per block row: 8, 4 or 2 (consecutive lanes)
    const int     ri   = s.gt / tpr;
    const int     ch   = s.gt - ri * tpr;
    double*       y    = s.y;
    T             e[kTrPre][VN];
    T             dv[DV][VN];
    // block bi's bounds: rows [b0, b0 + bw), solved columns [jlo, jhi)
    auto bounds = [&](int bi, int& b0, int& bw, int& jlo, int& jhi) {
        const int b = upper ? nblk - 1 - bi : bi;
        b0          = b * kBSolveNB;
        bw          = min(kBSolveNB, n - b0);
        jlo         = upper ? b0 + bw : 0;
        jhi         = upper ? n : b0;
    };
    auto prefetch = [&](int bi) {
        int b0, bw, jlo, jhi;
        bounds(bi, b0, bw, jlo, jhi);
        const int nvec = (jhi - jlo) / VN;
        const T*  row  = s.row(b0 + (ri < bw ? ri : 0));
#pragma unroll
        for (int u = 0; u < kTrPre; ++u)
        {
            const int m = ch + u * tpr;
            if (ri < bw && m < nvec)
            {
                vload(row + jlo + m * VN, e[u]);
            }
            else
            {
#pragma unroll
                for (int j = 0; j < VN; ++j)
                    e[u][j] = T(0);
            }
        }
#pragma unroll
        for (int u = 0; u < DV; ++u)
        {
            const int vv = ch + u * tpr;
            const int c  = b0 + vv * VN;
            if (ri < bw && vv < kBSolveNB / VN && c + VN <= n)
            {
                vload(row + c, dv[u]);
            }
            else
            {
#pragma unroll
                for (int j = 0; j < VN; ++j)
                    dv[u][j] = (ri < bw && vv < kBSolveNB / VN && c + j < n) ? row[c + j] : T(0);
            }
        }
    };
    prefetch(0);
    for (int bi = 0; bi < nblk; ++bi)
    {
        int b0, bw, jlo, jhi;
        bounds(bi, b0, bw, jlo, jhi);
        const int nvec = (jhi - jlo) / VN;
        double    acc  = 0.0;
        if (ri < bw)
        {
#pragma unroll
            for (int u = 0; u < DV; ++u)
            {
                const int vv = ch + u * tpr;
                if (vv < kBSolveNB / VN)
                {
#pragma unroll
                    for (int j = 0; j < VN; ++j)
                        s.dg[ri * kBDgLd + vv * VN + j] = dv[u][j];
                }
            }
            // four independent sums (a single chain of 64 dependent FP64
            // FMAs would set the pace)
            double a4[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int u = 0; u < kTrPre; ++u)
            {
                const int m = ch + u * tpr;
                if (m < nvec)
                {
#pragma unroll
                    for (int j = 0; j < VN; ++j)
                        a4[u & 3] = fma((double)e[u][j], y[jlo + m * VN + j], a4[u & 3]);
                }
            }
            acc = (a4[0] + a4[1]) + (a4[2] + a4[3]);
            // vectors past the prefetched ones, in batches of 8; then the
            // ragged tail
            const T* row = s.row(b0 + ri);
            for (int m0 = ch + kTrPre * tpr; m0 < nvec; m0 += 8 * tpr)
            {
                T f[8][VN];
#pragma unroll
                for (int u = 0; u < 8; ++u)
                {
                    const int m = m0 + u * tpr;
                    if (m < nvec)
                    {
                        vload(row + jlo + m * VN, f[u]);
                    }
                    else
                    {
#pragma unroll
                        for (int j = 0; j < VN; ++j)
                            f[u][j] = T(0);
                    }
                }
#pragma unroll
                for (int u = 0; u < 8; ++u)
                {
                    const int m = m0 + u * tpr;
                    if (m < nvec)
                    {
#pragma unroll
                        for (int j = 0; j < VN; ++j)
                            acc = fma((double)f[u][j], y[jlo + m * VN + j], acc);
                    }
                }
            }
            if (ch == 0)
            {
                for (int c = jlo + nvec * VN; c < jhi; ++c)
                    acc = fma((double)row[c], y[c], acc);
            }
        }
        for (int off = tpr >> 1; off > 0; off >>= 1)
        {
            acc += __shfl_xor_sync(0xffffffffu, acc, off);
        }
        if (ch == 0 && ri < bw)
        {
            s.dpart[ri] = acc;
        }
        if (bi + 1 < nblk)
        {
            prefetch(bi + 1);
        }
        s.sync();
        if (warp == 0)
        {
            double a[kBSolveNB];
#pragma unroll
            for (int j = 0; j < kBSolveNB; ++j)
            {
                a[j] = (lane < bw && j < bw) ? (double)s.dg[lane * kBDgLd + j] : 0.0;
            }
            double v = lane < bw ? y[b0 + lane] - s.dpart[lane] : 0.0;
            if (!upper)
            {
#pragma unroll
                for (int j = 0; j < kBSolveNB; ++j)
                {
                    const double yj = __shfl_sync(0xffffffffu, v, j);
                    if (lane > j && lane < bw && j < bw)
                    {
                        v = fma(-a[j], yj, v);
                    }
                }
            }
            else
            {
                const double rinv = lane < bw ? 1.0 / (double)s.dg[lane * kBDgLd + lane] : 0.0;
#pragma unroll
                for (int jj = 0; jj < kBSolveNB; ++jj)
                {
                    const int j = kBSolveNB - 1 - jj;
                    if (lane == j && j < bw)
                    {
                        v *= rinv;
                    }
                    const double yj = __shfl_sync(0xffffffffu, v, j);
                    if (lane < j && j < bw)
                    {
                        v = fma(-a[j], yj, v);
                    }
                }
            }
            if (lane < bw)
            {
                y[b0 + lane] = v;
            }
        }
        s.sync();
    }
}

// The rows the panel moved (sigma[r] != r: new local row r is old local row
// sigma[r]) take their new physical rows in the map: rowp[k + r] <-
// rowp[k + sigma[r]].  At most 2 nb rows move.  Ends with a group barrier.
template <typename T> __device__ void remap_rows(const Sys<T>& s, int k, int R)
{
    const int lane = s.gt & 31, warp = s.gt >> 5;
    int*      dst  = s.list;
    int*      old  = s.list + 2 * s.nb;
    if (warp == 0)
    {
        int cnt = 0;
        for (int r0 = 0; r0 < R; r0 += 32)
        {
            const int      r    = r0 + lane;
            const bool     mv   = r < R && s.sigma[r] != r;
            const unsigned bits = __ballot_sync(0xffffffffu, mv);
            if (mv)
            {
                const int q = cnt + __popc(bits & ((1u << lane) - 1u));
                dst[q]      = r;
                old[q]      = s.rowp[k + s.sigma[r]];
            }
            cnt += __popc(bits);
        }
        __syncwarp();
        for (int q = lane; q < cnt; q += 32)
        {
            s.rowp[k + dst[q]] = old[q];
        }
    }
    s.sync();
}

// Panel [k, k + w) x rows [k, n) in registers.  Rows never leave their
// thread: thread gt owns the panel's local rows gt + q G (q < RPT) and keeps
// each row's current position (the row order that partial pivoting's
// interchanges give, ties going to the lower position) in a register.  Per
// column: the pivot search over the rows at positions >= jj (redux.sync per
// warp, then over the warps), the pivot row posted to shared memory, and the
// update of every row not yet a pivot.  The column loop is not unrolled (the
// code of 32 unrolled columns outgrows the instruction cache): every row's
// registers rotate left by one per column, so the active column is always
// register 0 and the column just finished (a multiplier, or the pivot row's
// own value) moves to the end; after NB rotations each row is back in
// column order: multipliers, then (for a pivot row) its row of U.
// On return: the map is updated, the factor rows are written back, P holds
// L11 (positions < w) and LT holds L21^T.
template <typename T, int NB, int RPT> __device__ void panel_regs(const Sys<T>& s, int k, int w)
{
    using K            = typename BKey<T>::type;
    constexpr int VN   = 16 / (int)sizeof(T);
    const int     n    = s.n;
    const int     R    = n - k;
    const int     lane = s.gt & 31, warp = s.gt >> 5, warps = s.G >> 5;
    const int     ldp  = s.nb + 1;
    T*            urow = s.dg;  // the pivot row, active column first (16-byte aligned)
    T             v[RPT][NB];
    int           pos[RPT];
    bool          live[RPT];    // a row of the panel that is not yet a pivot
#pragma unroll
    for (int q = 0; q < RPT; ++q)
    {
        const int r = s.gt + q * s.G;
        pos[q]      = r;
        live[q]     = r < R;
        if (r < R)
        {
            const T* src = s.row(k + r) + k;
            if (w == NB)
            {
#pragma unroll
                for (int c = 0; c < NB; c += VN)
                    vload(src + c, &v[q][c]);
            }
            else
            {
#pragma unroll
                for (int c = 0; c < NB; ++c)
                    v[q][c] = c < w ? src[c] : T(0);
            }
        }
        else
        {
#pragma unroll
            for (int c = 0; c < NB; ++c)
                v[q][c] = T(0);
        }
    }
#pragma unroll 1
    for (int jj = 0; jj < NB; ++jj)
    {
        if (jj < w)
        {
            K   ck = 0;
            int cr = INT_MAX;
#pragma unroll
            for (int q = 0; q < RPT; ++q)
            {
                if (live[q])
                {
                    const K key = bkey(v[q][0], pos[q] == jj);
                    if (key > ck || (key == ck && pos[q] < cr))
                    {
                        ck = key;
                        cr = pos[q];
                    }
                }
            }
            bwarp_best(ck, cr);
            if (lane == 0)
            {
                s.red_key[warp] = (unsigned long long)ck;
                s.red_row[warp] = cr;
            }
            s.sync();
            K   pk = lane < warps ? (K)s.red_key[lane] : K(0);
            int p  = lane < warps ? s.red_row[lane] : INT_MAX;
            bwarp_best(pk, p);
            // position jj holds a live row, so p is a position of the panel
#pragma unroll
            for (int q = 0; q < RPT; ++q)
            {
                if (live[q] && pos[q] == p)
                {
#pragma unroll
                    for (int c = 0; c < NB; c += VN)
                        vstore(urow + c, &v[q][c]);
                }
            }
            s.sync();
            const T d = urow[0];
            if (d == T(0) && s.gt == 0 && s.flags[0] < 0)
            {
                s.flags[0] = k + jj;
            }
            // the interchange of positions jj and p
#pragma unroll
            for (int q = 0; q < RPT; ++q)
            {
                if (live[q] && pos[q] == p)
                {
                    live[q] = false;
                    pos[q]  = jj;
                }
                else if (live[q] && pos[q] == jj)
                {
                    pos[q] = p;
                }
            }
            T u[NB];
#pragma unroll
            for (int c = 0; c < NB; c += VN)
                vload(urow + c, &u[c]);
            const int lim = NB - jj;  // registers [1, lim) hold the columns still to update
#pragma unroll
            for (int q = 0; q < RPT; ++q)
            {
                if (live[q] && d != T(0))
                {
                    const T l = v[q][0] / d;
                    v[q][0]   = l;
#pragma unroll
                    for (int c = 1; c < NB; ++c)
                    {
                        if (c < lim)
                            v[q][c] = fma(-l, u[c], v[q][c]);
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < RPT; ++q)
        {
            const T t = v[q][0];
#pragma unroll
            for (int c = 0; c < NB - 1; ++c)
                v[q][c] = v[q][c + 1];
            v[q][NB - 1] = t;
        }
    }
    // write back (the rows' physical places do not change), L11 into P,
    // L21^T into LT, and the final order into sigma for the map
#pragma unroll
    for (int q = 0; q < RPT; ++q)
    {
        const int r = s.gt + q * s.G;
        if (r < R)
        {
            T* dst = s.row(k + r) + k;
            if (w == NB)
            {
#pragma unroll
                for (int c = 0; c < NB; c += VN)
                    vstore(dst + c, &v[q][c]);
            }
            else
            {
#pragma unroll
                for (int c = 0; c < NB; ++c)
                    if (c < w)
                        dst[c] = v[q][c];
            }
            const int ps = pos[q];
            if (ps < w)
            {
#pragma unroll
                for (int c = 0; c < NB; ++c)
                    if (c < w)
                        s.P[ps * ldp + c] = v[q][c];
            }
            else
            {
#pragma unroll
                for (int c = 0; c < NB; ++c)
                    if (c < w)
                        s.LT[c * s.np + (ps - w)] = v[q][c];
            }
            s.sigma[ps] = r;
        }
    }
    s.sync();
    remap_rows(s, k, R);
}

// The same panel in shared memory (P), for orders whose rows do not fit the
// register panel's rows per thread.
template <typename T> __device__ void panel_smem(const Sys<T>& s, int k, int w)
{
    using K        = typename BKey<T>::type;
    const int n    = s.n;
    const int R    = n - k;
    const int lane = s.gt & 31, warp = s.gt >> 5, warps = s.G >> 5;
    const int ldp  = s.nb + 1;
    // load: 4 elements in flight per thread
    for (int e0 = s.gt; e0 < R * w; e0 += 4 * s.G)
    {
        T   t[4];
        int rr[4], cc[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
        {
            const int e = e0 + u * s.G;
            rr[u]       = e / w;
            cc[u]       = e - rr[u] * w;
            t[u]        = e < R * w ? s.row(k + rr[u])[k + cc[u]] : T(0);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
        {
            if (e0 + u * s.G < R * w)
                s.P[rr[u] * ldp + cc[u]] = t[u];
        }
    }
    for (int r = s.gt; r < R; r += s.G)
    {
        s.sigma[r] = r;
    }
    s.sync();
    K   ck = 0;
    int cr = INT_MAX;
    for (int r = s.gt; r < R; r += s.G)
    {
        const K key = bkey(s.P[r * ldp], r == 0);
        if (key > ck)
        {
            ck = key;
            cr = r;
        }
    }
    for (int jj = 0; jj < w; ++jj)
    {
        bwarp_best(ck, cr);
        if (lane == 0)
        {
            s.red_key[warp] = (unsigned long long)ck;
            s.red_row[warp] = cr;
        }
        s.sync();
        K   pk = lane < warps ? (K)s.red_key[lane] : K(0);
        int p  = lane < warps ? s.red_row[lane] : INT_MAX;
        bwarp_best(pk, p);
        if (p != jj)
        {
            for (int c = s.gt; c < w; c += s.G)
            {
                const T t         = s.P[jj * ldp + c];
                s.P[jj * ldp + c] = s.P[p * ldp + c];
                s.P[p * ldp + c]  = t;
            }
        }
        if (s.gt == 0 && p != jj)
        {
            const int t = s.sigma[jj];
            s.sigma[jj] = s.sigma[p];
            s.sigma[p]  = t;
        }
        s.sync();
        const T d = s.P[jj * ldp + jj];
        if (d == T(0) && s.gt == 0 && s.flags[0] < 0)
        {
            s.flags[0] = k + jj;
        }
        ck = 0;
        cr = INT_MAX;
        for (int r = jj + 1 + s.gt; r < R; r += s.G)
        {
            T* row = s.P + r * ldp;
            if (d != T(0))
            {
                const T l = row[jj] / d;
                row[jj]   = l;
                for (int c = jj + 1; c < w; ++c)
                {
                    row[c] = fma(-l, s.P[jj * ldp + c], row[c]);
                }
            }
            if (jj + 1 < w)
            {
                const K key = bkey(row[jj + 1], r == jj + 1);
                if (key > ck)
                {
                    ck = key;
                    cr = r;
                }
            }
        }
    }
    s.sync();
    remap_rows(s, k, R);
    for (int e = s.gt; e < R * w; e += s.G)
    {
        const int r         = e / w, c = e - r * w;
        const T   t         = s.P[r * ldp + c];
        s.row(k + r)[k + c] = t;
        if (r >= w)
        {
            s.LT[c * s.np + (r - w)] = t;
        }
    }
    s.sync();
}

// A22 -= L21 U12 for the rows and columns [k + w, n): TM x 8 tiles per
// thread, (G / 16) TM rows x 128 columns per pass; a thread's 8 columns are
// two 4-column halves 64 apart, so that the 16 threads of a row read U12 in
// one contiguous 256-byte run.  The tile of A22 is loaded before the product
// so that its latency hides behind the w rank-1 steps.
template <typename T> __device__ void trailing_update(const Sys<T>& s, int k, int w, int rest)
{
    constexpr int TM = BatchTraits<T>::TM;
    constexpr int VN = 16 / (int)sizeof(T);
    constexpr int HN = 4;  // columns per half
    const int     tx = s.gt & 15, ty = s.gt >> 4;
    const int     th = (s.G >> 4) * TM;
    const int     c0 = k + w;
    for (int i0 = 0; i0 < rest; i0 += th)
    {
        for (int j0 = 0; j0 < rest; j0 += 128)
        {
            const int ri  = i0 + ty * TM;
            const int cl  = j0 + tx * HN;
            const int chi = cl + 64;
            if (ri >= rest || cl >= rest)
            {
                continue;
            }
            const bool hi = chi < rest;
            T          c[TM][2 * HN];
#pragma unroll
            for (int a = 0; a < TM; ++a)
            {
#pragma unroll
                for (int h = 0; h < 2; ++h)
                {
                    const int col = h ? chi : cl;
                    if (ri + a < rest && (h == 0 || hi))
                    {
                        const T* src = s.row(c0 + ri + a) + c0 + col;
                        if (col + HN <= rest)
                        {
#pragma unroll
                            for (int j = 0; j < HN; j += VN)
                                vload(src + j, &c[a][h * HN + j]);
                        }
                        else
                        {
#pragma unroll
                            for (int j = 0; j < HN; ++j)
                                c[a][h * HN + j] = col + j < rest ? src[j] : T(0);
                        }
                    }
                    else
                    {
#pragma unroll
                        for (int j = 0; j < HN; ++j)
                            c[a][h * HN + j] = T(0);
                    }
                }
            }
            T acc[TM][2 * HN];
#pragma unroll
            for (int a = 0; a < TM; ++a)
#pragma unroll
                for (int b = 0; b < 2 * HN; ++b)
                    acc[a][b] = T(0);
#pragma unroll 4
            for (int kk = 0; kk < w; ++kk)
            {
                T        lv[TM], uv[2 * HN];
                const T* lt = s.LT + kk * s.np + ri;
                const T* ut = s.U + kk * s.np;
#pragma unroll
                for (int a = 0; a < TM; a += VN)
                    vload(lt + a, &lv[a]);
#pragma unroll
                for (int j = 0; j < HN; j += VN)
                    vload(ut + cl + j, &uv[j]);
                if (hi)
                {
#pragma unroll
                    for (int j = 0; j < HN; j += VN)
                        vload(ut + chi + j, &uv[HN + j]);
                }
                else
                {
#pragma unroll
                    for (int j = 0; j < HN; ++j)
                        uv[HN + j] = T(0);
                }
#pragma unroll
                for (int a = 0; a < TM; ++a)
#pragma unroll
                    for (int b = 0; b < 2 * HN; ++b)
                        acc[a][b] = fma(lv[a], uv[b], acc[a][b]);
            }
#pragma unroll
            for (int a = 0; a < TM; ++a)
            {
                if (ri + a >= rest)
                {
                    continue;
                }
#pragma unroll
                for (int h = 0; h < 2; ++h)
                {
                    const int col = h ? chi : cl;
                    if (h == 1 && !hi)
                    {
                        continue;
                    }
                    T out[HN];
#pragma unroll
                    for (int j = 0; j < HN; ++j)
                        out[j] = c[a][h * HN + j] - acc[a][h * HN + j];
                    T* dst = s.row(c0 + ri + a) + c0 + col;
                    if (col + HN <= rest)
                    {
#pragma unroll
                        for (int j = 0; j < HN; j += VN)
                            vstore(dst + j, &out[j]);
                    }
                    else
                    {
#pragma unroll
                        for (int j = 0; j < HN; ++j)
                            if (col + j < rest)
                                dst[j] = out[j];
                    }
                }
            }
        }
    }
}

template <typename T, int NB> __device__ void lu_factor_nb(const Sys<T>& s)
{
    const int n   = s.n;
    const int ldp = NB + 1;
    const int rpt = panel_rpt<T>(n, NB, s.G);
    for (int k = 0; k < n; k += NB)
    {
        const int w    = min(NB, n - k);
        const int rest = n - k - w;
        // ---- the panel: factored, rows remapped, written back; L11 in P,
        // L21^T in LT
        if (rpt == 2)
        {
            panel_regs<T, NB, 2>(s, k, w);
        }
        else
        {
            if constexpr (4 * NB * sizeof(T) <= 256)
            {
                if (rpt == 4)
                    panel_regs<T, NB, 4>(s, k, w);
                else
                    panel_smem(s, k, w);
            }
            else
            {
                panel_smem(s, k, w);
            }
        }
        B200LA_BPHASE(1);
        if (rest <= 0)
        {
            break;
        }
        // ---- U12 = L11^-1 A12 (thread per column)
        for (int c = s.gt; c < rest; c += s.G)
        {
            T u[NB];
#pragma unroll
            for (int i = 0; i < NB; ++i)
            {
                u[i] = i < w ? s.row(k + i)[k + w + c] : T(0);
            }
#pragma unroll
            for (int i = 1; i < NB; ++i)
            {
#pragma unroll
                for (int j = 0; j < i; ++j)
                {
                    u[i] = fma(-s.P[i * ldp + j], u[j], u[i]);
                }
            }
#pragma unroll
            for (int i = 0; i < NB; ++i)
            {
                if (i < w)
                {
                    s.row(k + i)[k + w + c] = u[i];
                    s.U[i * s.np + c]       = u[i];
                }
            }
        }
        s.sync();
        B200LA_BPHASE(2);
        trailing_update(s, k, w, rest);
        s.sync();
        B200LA_BPHASE(3);
    }
}

template <typename T> __device__ void lu_factor(const Sys<T>& s)
{
    if (s.nb == BatchTraits<T>::kMaxNB)
        lu_factor_nb<T, BatchTraits<T>::kMaxNB>(s);
    else
        lu_factor_nb<T, BatchTraits<T>::kMinNB>(s);
}

// Rows [i0, i0 + 2) of A (FP64, row-major n x n), a warp's lanes over the
// columns: both rows' loads are issued before any is used.
constexpr int kBPerLane = kBMaxN / 32;
__device__ __forceinline__ void load_two_rows(const double* __restrict__ a, int n, int i0, int lane,
    double (&e)[2][kBPerLane])
{
#pragma unroll
    for (int h = 0; h < 2; ++h)
    {
#pragma unroll
        for (int m = 0; m < kBPerLane; ++m)
        {
            const int j = lane + 32 * m;
            e[h][m]     = (i0 + h < n && j < n) ? a[(size_t)(i0 + h) * n + j] : 0.0;
        }
    }
}

template <typename T>
__device__ void solve_system(Sys<T>& s, const double* __restrict__ a, const double* __restrict__ b,
    double* __restrict__ x, int max_iter, double tol, bool fallback, int32_t* status, double* berr, int sys)
{
    const int n     = s.n;
    const int lane  = s.gt & 31, warp = s.gt >> 5;
    const int warps = s.G >> 5;
    if (s.gt == 0)
    {
        s.flags[0] = -1;
    }
    for (int i = s.gt; i < n; i += s.G)
    {
        s.rowp[i] = i;
    }
    // ---- A -> F in T, ||A||_inf: a warp per row, two rows in flight; the
    // norm lands in y[0..warps)
    double anorm = 0.0;
    for (int i0 = 2 * warp; i0 < n; i0 += 2 * warps)
    {
        double e[2][kBPerLane];
        load_two_rows(a, n, i0, lane, e);
#pragma unroll
        for (int h = 0; h < 2; ++h)
        {
            if (i0 + h >= n)
            {
                continue;
            }
            T*     dst = s.f + (size_t)(i0 + h) * s.ld;
            double acc = 0.0;
#pragma unroll
            for (int m = 0; m < kBPerLane; ++m)
            {
                const int j = lane + 32 * m;
                if (j < n)
                {
                    dst[j] = (T)e[h][m];
                    acc += fabs(e[h][m]);
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1)
            {
                acc += __shfl_xor_sync(0xffffffffu, acc, off);
            }
            anorm = fmax(anorm, acc);
        }
    }
    if (lane == 0)
    {
        s.y[warp] = anorm;
    }
    s.sync();
    anorm = 0.0;
    for (int q = 0; q < warps; ++q)
    {
        anorm = fmax(anorm, s.y[q]);
    }
    s.sync();
    B200LA_BPHASE(0);
    lu_factor(s);
    if (s.flags[0] >= 0)
    {
        if (s.gt == 0)
        {
            status[sys] = -(s.flags[0] + 1);
            berr[sys]   = INFINITY;
        }
        s.sync();
        return;
    }
    double bnorm = 0.0;
    for (int i = s.gt; i < n; i += s.G)
    {
        s.x[i] = 0.0;
        s.r[i] = b[i];
    }
    s.sync();
    for (int i = 0; i < n; ++i)
    {
        bnorm = fmax(bnorm, fabs(s.r[i]));
    }
    int    it       = 0;
    double eta      = INFINITY;
    double eta_prev = INFINITY;
    bool   done     = false;
    for (;;)
    {
        // the factor's logical row i is A's row rowp[i]
        for (int i = s.gt; i < n; i += s.G)
        {
            s.y[i] = s.r[s.rowp[i]];
        }
        s.sync();
        bat_trsv(s, false);
        bat_trsv(s, true);
        for (int i = s.gt; i < n; i += s.G)
        {
            s.x[i] += s.y[i];
        }
        s.sync();
        B200LA_BPHASE(4);
        // r = b - A x (a warp per row, two rows in flight), max|r|, max|x|
        double rmax = 0.0, xmax = 0.0;
        for (int i0 = 2 * warp; i0 < n; i0 += 2 * warps)
        {
            double e[2][kBPerLane];
            load_two_rows(a, n, i0, lane, e);
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                double acc = 0.0;
#pragma unroll
                for (int m = 0; m < kBPerLane; ++m)
                {
                    const int j = lane + 32 * m;
                    if (j < n)
                    {
                        acc = fma(e[h][m], s.x[j], acc);
                    }
                }
#pragma unroll
                for (int off = 16; off > 0; off >>= 1)
                {
                    acc += __shfl_xor_sync(0xffffffffu, acc, off);
                }
                const int i = i0 + h;
                if (lane == 0 && i < n)
                {
                    const double ri = b[i] - acc;
                    s.r[i]          = ri;
                    rmax            = fmax(rmax, fabs(ri));
                    xmax            = fmax(xmax, fabs(s.x[i]));
                }
            }
        }
        if (lane == 0)
        {
            s.y[2 * warp]     = rmax;
            s.y[2 * warp + 1] = xmax;
        }
        s.sync();
        rmax = xmax = 0.0;
        for (int q = 0; q < warps; ++q)
        {
            rmax = fmax(rmax, s.y[2 * q]);
            xmax = fmax(xmax, s.y[2 * q + 1]);
        }
        s.sync();
        B200LA_BPHASE(5);
        const double den = anorm * xmax + bnorm;
        eta              = den > 0 ? rmax / den : 0.0;
        ++it;
        if (eta <= tol)
        {
            done = true;
            break;
        }
        // out of corrections, not a number, or stalled (less than a factor 2
        // gained after the first correction)
        if (it > max_iter || !(eta == eta) || (it > 2 && eta > 0.5 * eta_prev))
        {
            break;
        }
        eta_prev = eta;
    }
    for (int i = s.gt; i < n; i += s.G)
    {
        x[i] = s.x[i];
    }
    if (s.gt == 0)
    {
        status[sys] = done ? (fallback ? kEscalated + it - 1 : it - 1) : kNotConverged;
        berr[sys]   = eta;
    }
    s.sync();
}

template <typename T>
__global__ void __launch_bounds__(kBT, 1) k_batched_gesv(int count, const int32_t* __restrict__ sizes,
    const int64_t* __restrict__ offa, const int64_t* __restrict__ offv, const int32_t* __restrict__ order,
    const double* __restrict__ A, const double* __restrict__ B, double* __restrict__ X, T* __restrict__ F,
    int max_iter, double tol, int fallback_only, const int32_t* __restrict__ table, int32_t* __restrict__ status,
    double* __restrict__ berr, int32_t* __restrict__ queue)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_sys[kBT / 64];
    __shared__ int s_g, s_nb, s_rounds;
    const int tid = threadIdx.x;
    auto entry_of = [&](int n) {
        return table != nullptr ? table[min((n - 1) / 64, kBBuckets - 1)] : BatchTraits<T>::kMaxNB;
    };
    T* slot = F + (size_t)blockIdx.x * (kBScratch / sizeof(T));
    for (;;)
    {
        // the CTA's next chunk: the first system sets the group size and
        // panel width; one more system per further group
        if (tid == 0)
        {
            const int q0 = atomicAdd(queue, 1);
            s_g          = 0;
            s_rounds     = 1;
            if (q0 < count)
            {
                const int sys0 = order != nullptr ? order[q0] : q0;
                const int e    = entry_of(sizes[sys0]);
                int       G    = entry_g(e);
                int       nb   = entry_nb(e);
                nb             = nb_supported<T>(nb) ? nb : BatchTraits<T>::kMaxNB;
                s_sys[0]       = sys0;
                bool fits      = group_fits<T>(sizes[sys0], nb, G);
                for (int g = 1; g < kBT / G; ++g)
                {
                    const int q = atomicAdd(queue, 1);
                    s_sys[g]    = q < count ? (order != nullptr ? order[q] : q) : -1;
                    if (s_sys[g] >= 0 && !group_fits<T>(sizes[s_sys[g]], nb, G))
                    {
                        fits = false;  // a larger system than the first (an unsorted order)
                    }
                }
                if (!fits)
                {
                    // the chunk's systems one after another with the whole CTA
                    s_rounds = kBT / G;
                    G        = kBT;
                }
                s_g  = G;
                s_nb = nb;
            }
        }
        __syncthreads();
        const int G = s_g;
        if (G == 0)
        {
            return;
        }
        for (int round = 0; round < s_rounds; ++round)
        {
            const int group = tid / G;
            const int sys   = s_sys[s_rounds > 1 ? round : group];
            if (sys >= 0 && !(fallback_only && status[sys] != kNotConverged))
            {
                Sys<T> s;
                s.n                  = sizes[sys];
                s.nb                 = s_nb;
                s.G                  = G;
                s.gt                 = tid - group * G;
                s.bar                = 1 + group;
                s.ld                 = bat_ld<T>(s.n);
                s.f                  = slot + (size_t)group * (group_scratch_bytes(G) / sizeof(T));
                s.np                 = group_np(s.n);
                const GroupSmem L    = group_layout<T>(s.n, s.nb, G);
                unsigned char*  base = smem_raw + (size_t)group * group_smem_bytes(G);
                s.P                  = reinterpret_cast<T*>(base + L.P);
                s.LT                 = reinterpret_cast<T*>(base + L.LT);
                s.U                  = reinterpret_cast<T*>(base + L.U);
                s.y                  = reinterpret_cast<double*>(base + L.y);
                s.r                  = reinterpret_cast<double*>(base + L.r);
                s.x                  = reinterpret_cast<double*>(base + L.x);
                s.dg                 = reinterpret_cast<T*>(base + L.dg);
                s.dpart              = reinterpret_cast<double*>(base + L.dpart);
                s.sigma              = reinterpret_cast<int*>(base + L.sigma);
                s.list               = reinterpret_cast<int*>(base + L.list);
                s.rowp               = reinterpret_cast<int*>(base + L.rowp);
                s.red_key            = reinterpret_cast<unsigned long long*>(base + L.red);
                s.red_row            = reinterpret_cast<int*>(base + L.red + 64);
                s.flags              = reinterpret_cast<int*>(base + L.red + 64 + 32);
                solve_system(s, A + offa[sys], B + offv[sys], X + offv[sys], max_iter, tol, fallback_only != 0,
                    status, berr, sys);
            }
            __syncthreads();
        }
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
        (int)kBatchedSmem));
    if (dev >= 0 && dev < 64)
        done[dev] = true;
    return B200LA_SUCCESS;
}

// Whether the largest order of every bucket fits its group (shared-memory
// slice and factor scratch) with the bucket's panel width, and every panel
// width is one the kernel is built for (the systems are taken largest
// first, so a group never gets a larger one than its chunk's first).
template <typename T> bool table_fits(const int32_t* table_host)
{
    for (int bk = 0; bk < kBBuckets; ++bk)
    {
        const int e  = table_host[bk];
        const int G  = entry_g(e);
        const int nb = entry_nb(e);
        if (!nb_supported<T>(nb))
            return false;
        const int nmax = bk == kBBuckets - 1 ? kBMaxN : 64 * (bk + 1);
        if (!group_fits<T>(nmax, nb, G))
            return false;
    }
    return true;
}

// Factor-scratch slots for a batch of at most `systems` systems.
inline int64_t scratch_slots(int64_t systems) { return systems < kBMaxCTAs ? systems : kBMaxCTAs; }
}  // namespace
int require_sm100();
}  // namespace b200la

using namespace b200la;

extern "C" {

B200LA_API size_t b200la_dgesv_batched_workspace_size(int64_t total_a, int64_t total_v, int precision)
{
    (void)precision;
    if (total_a <= 0 || total_v <= 0)
        return 0;
    Arena a;
    a.next<int32_t>(64);  // queue counters of the two passes
    // factor scratch: one slot per CTA (a batch has at most total_v
    // systems); the FP32 and the FP64 pass use the same slots
    a.next<unsigned char>((size_t)scratch_slots(total_v) * kBScratch);
    return a.size();
}

B200LA_API int b200la_batched_table_valid(int precision, const int32_t* table_host)
{
    if (table_host == nullptr)
        return 0;
    return precision == B200LA_PREC_FP64 ? (table_fits<double>(table_host) ? 1 : 0)
                                         : (table_fits<float>(table_host) ? 1 : 0);
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
    if (count > total_v)
        return set_error(B200LA_INVALID_ARGUMENT, "dgesv_batched: more systems than right-hand-side values");
    const size_t need = b200la_dgesv_batched_workspace_size(total_a, total_v, precision);
    if (workspace == nullptr || workspace_bytes < need)
        return set_error(B200LA_WORKSPACE_TOO_SMALL, "dgesv_batched: workspace too small (%zu < %zu)",
            workspace_bytes, need);
    int rc = require_sm100();
    if (rc != B200LA_SUCCESS)
        return rc;
    cudaStream_t  s     = static_cast<cudaStream_t>(stream);
    Arena         ar(workspace, workspace_bytes);
    int32_t*      queue = ar.next<int32_t>(64);
    const int64_t slots = scratch_slots(total_v);
    const int64_t sms   = device_sm_count();
    const int     grid  = (int)(sms < slots ? sms : slots);
    B200LA_CUDA(cudaMemsetAsync(queue, 0, sizeof(int32_t) * 2, s));
    void* fbuf = ar.next<unsigned char>((size_t)slots * kBScratch);
    if ((rc = set_batched_attr<double>()) != B200LA_SUCCESS)
        return rc;
    if (precision == B200LA_PREC_FP64)
    {
        prof_begin(KC_BATCHED, s);
        k_batched_gesv<double><<<grid, kBT, kBatchedSmem, s>>>((int)count, sizes, offsets_a, offsets_v, order, a, b,
            x, (double*)fbuf, max_iterations, tolerance, 0, nb_table, status, backward_error, queue);
        prof_end(KC_BATCHED, s);
    }
    else
    {
        if ((rc = set_batched_attr<float>()) != B200LA_SUCCESS)
            return rc;
        prof_begin(KC_BATCHED, s);
        k_batched_gesv<float><<<grid, kBT, kBatchedSmem, s>>>((int)count, sizes, offsets_a, offsets_v, order, a, b,
            x, (float*)fbuf, max_iterations, tolerance, 0, nb_table, status, backward_error, queue);
        prof_end(KC_BATCHED, s);
        B200LA_LAUNCH_CHECK();
        // FP64 factors for the systems whose FP32 refinement stalled (one
        // system per CTA, panel width 16)
        prof_begin(KC_BATCHED, s);
        k_batched_gesv<double><<<grid, kBT, kBatchedSmem, s>>>((int)count, sizes, offsets_a, offsets_v, order, a, b,
            x, (double*)fbuf, 3, tolerance, 1, nullptr, status, backward_error, queue + 1);
        prof_end(KC_BATCHED, s);
    }
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}
}
