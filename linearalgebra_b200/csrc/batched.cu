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
//   * A (FP64, global) is copied into the factor buffer in the
//     factorization type T (float: FP32 factors + FP64 refinement; double:
//     plain FP64 LU), with ||A||_inf on the way;
//   * blocked right-looking LU with partial pivoting, panel width NB:
//       - the panel (all remaining rows x NB columns) is factored in shared
//         memory: per column a pivot search (integer keys, redux.sync), the
//         row swap inside the panel and the rank-1 update with the next
//         column's pivot search fused into it;
//       - the panel's interchanges are composed into one permutation of the
//         rows they touch and applied to the other columns as one gather
//         (staged in shared memory) and one scatter;
//       - U12 = L11^-1 A12, one thread per column, in shared memory;
//       - A22 -= L21 U12 with 8 x 8 (FP32) or 4 x 8 (FP64) register tiles per
//         thread, L21 (transposed) and U12 from shared memory;
//   * the solve applies the factors in FP64: 32-row blocks, the diagonal
//     block in one warp's registers (rows by lane, substitution with
//     shuffles), the other rows updated by every thread; then FP64 refinement
//     r = b - A x, d = U^-1 L^-1 P r, x += d until the normwise backward
//     error ||r|| / (||A|| ||x|| + ||b||) <= tol, the refinement stalls (less
//     than a factor 2 gained per correction after the first) or max_iter
//     corrections.
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

namespace b200la
{
namespace
{
constexpr int kBT       = 256;  // threads per CTA
constexpr int kBMaxN    = 512;
constexpr int kBBuckets = 8;    // order buckets of 64
constexpr int kBSolveNB = 32;   // rows per block of the triangular solves
// status of a system whose refinement stalled or ran out of corrections; the
// FP64 pass picks these up.  Systems finished by that pass get 1000 + k.
constexpr int32_t kNotConverged = -1000000;
constexpr int32_t kEscalated    = 1000;

template <typename T> struct BatchTraits;
template <> struct BatchTraits<float>
{
    static constexpr int kMaxNB = 32;
    static constexpr int TM     = 8;  // rows of a thread's update tile
    static constexpr int TN     = 8;  // columns
};
template <> struct BatchTraits<double>
{
    static constexpr int kMaxNB = 16;
    static constexpr int TM     = 4;
    static constexpr int TN     = 8;
};

// A bucket's table entry: bits 0-7 the panel width NB, bits 8-15 the
// threads per system / 32 (0: the whole CTA).
__host__ __device__ inline int entry_nb(int e) { return e & 0xff; }
__host__ __device__ inline int entry_g(int e)
{
    const int g = ((e >> 8) & 0xff) * 32;
    return g == 64 || g == 128 ? g : kBT;
}

__host__ __device__ inline int group_np(int n) { return (n + 7) / 8 * 8 + 8; }

// Shared-memory slice of one group solving a system of order n with panel
// width nb (the same function sizes and carves).
struct GroupSmem
{
    size_t P, LT, U, y, r, x, sigma, list, piv, perm, red, end;
};
template <typename T> __host__ __device__ inline GroupSmem group_layout(int n, int nb)
{
    auto up = [](size_t v) { return (v + 15) / 16 * 16; };
    const int np = group_np(n);              // padded rows of LT and U (the update tiles read past n)
    const int nv = n > 16 ? n : 16;          // FP64 vectors (also the group's reductions: 2 per warp)
    GroupSmem g;
    g.P     = 0;                                                   // T[n][nb + 1]: the panel
    g.LT    = up(g.P + sizeof(T) * (size_t)n * (nb + 1));          // T[nb][np]: L21 transposed / staging
    g.U     = up(g.LT + sizeof(T) * (size_t)nb * np);              // T[nb][np]: U12
    g.y     = up(g.U + sizeof(T) * (size_t)nb * np);               // double[nv]
    g.r     = up(g.y + sizeof(double) * nv);                       // double[nv]
    g.x     = up(g.r + sizeof(double) * nv);                       // double[nv]
    g.sigma = up(g.x + sizeof(double) * nv);                       // int[n]: composed panel permutation
    g.list  = up(g.sigma + sizeof(int) * n);                       // int[2][2 nb]: rows it moves
    g.piv   = up(g.list + sizeof(int) * 4 * nb);                   // int[n]: pivot row of each step
    g.perm  = up(g.piv + sizeof(int) * n);                         // int[n]: final row permutation
    g.red   = up(g.perm + sizeof(int) * n);                        // 8 x (u64 key, int row) + flags
    g.end   = up(g.red + 8 * 8 + 8 * 4 + 64);
    return g;
}

constexpr size_t kBatchedSmem = 227 * 1024 - 1024;  // dynamic shared memory per CTA

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

// One group's state for one system.
template <typename T> struct Sys
{
    int      n, nb, G, gt, bar;  // order, panel width, threads, this thread's index, barrier id
    T*       f;                  // factor buffer (global), n x n row-major
    T*       P;                  // [n][nb + 1]
    T*       LT;                 // [nb][np]
    T*       U;                  // [nb][np]
    int      np;
    double * y, *r, *x;
    int *    sigma, *list, *piv, *perm;
    unsigned long long* red_key;
    int*                red_row;
    int*                flags;  // [0] first zero pivot (-1 none), [1] list count, [2] pivot of the column

    __device__ void sync() const { group_sync(bar, G); }
};

// y <- T^-1 y for the unit-lower (upper = false) or upper triangle of the
// factor (FP64 arithmetic).  32-row blocks in solve order: warp 0 of the group
// holds the diagonal block in registers (row b0 + lane) and substitutes with
// shuffles; then every thread updates its rows not yet solved.
template <typename T> __device__ void bat_trsv(const Sys<T>& s, bool upper)
{
    const int lane = s.gt & 31, warp = s.gt >> 5;
    const int n    = s.n;
    const int nblk = (n + kBSolveNB - 1) / kBSolveNB;
    double*   y    = s.y;
    for (int bi = 0; bi < nblk; ++bi)
    {
        const int b  = upper ? nblk - 1 - bi : bi;
        const int b0 = b * kBSolveNB;
        const int bw = min(kBSolveNB, n - b0);
        if (warp == 0)
        {
            double a[kBSolveNB];
            const T* row = s.f + (size_t)(b0 + (lane < bw ? lane : 0)) * n + b0;
#pragma unroll
            for (int j = 0; j < kBSolveNB; ++j)
            {
                a[j] = (lane < bw && j < bw) ? (double)row[j] : 0.0;
            }
            double v = lane < bw ? y[b0 + lane] : 0.0;
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
#pragma unroll
                for (int jj = 0; jj < kBSolveNB; ++jj)
                {
                    const int j = kBSolveNB - 1 - jj;
                    if (lane == j && j < bw)
                    {
                        v = v / a[j];
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
        for (int i = s.gt; i < n; i += s.G)
        {
            if (upper ? i < b0 : i >= b0 + bw)
            {
                const T* row = s.f + (size_t)i * n + b0;
                double   acc = 0.0;
#pragma unroll 8
                for (int j = 0; j < bw; ++j)
                {
                    acc = fma((double)row[j], y[b0 + j], acc);
                }
                y[i] -= acc;
            }
        }
        s.sync();
    }
}

// The panel's interchanges (sigma: new row r of the block [k, n) is old row
// sigma[r]) on columns [c0, c1) of the factor, for the `cnt` rows in the
// list: values gathered into the LT buffer (cnt x 32 columns at a time),
// then scattered.
template <typename T> __device__ void apply_interchanges(const Sys<T>& s, int k, int cnt, int c0, int c1)
{
    const int* dst = s.list;
    const int* src = s.list + 2 * s.nb;
    // staging in the LT and U buffers (2 nb x np elements; cnt <= np rows of
    // 2 nb columns per round)
    T*        stg = s.LT;
    const int cwp = 2 * s.nb;
    for (int cb = c0; cb < c1; cb += cwp)
    {
        const int cw = min(cwp, c1 - cb);
        for (int e = s.gt; e < cnt * cwp; e += s.G)
        {
            const int q = e / cwp, c = e - q * cwp;
            if (c < cw)
            {
                stg[e] = s.f[(size_t)(k + src[q]) * s.n + cb + c];
            }
        }
        s.sync();
        for (int e = s.gt; e < cnt * cwp; e += s.G)
        {
            const int q = e / cwp, c = e - q * cwp;
            if (c < cw)
            {
                s.f[(size_t)(k + dst[q]) * s.n + cb + c] = stg[e];
            }
        }
        s.sync();
    }
}

template <typename T> __device__ void lu_factor(const Sys<T>& s)
{
    using K             = typename BKey<T>::type;
    constexpr int TM    = BatchTraits<T>::TM;
    constexpr int TN    = BatchTraits<T>::TN;
    const int     n     = s.n;
    const int     lane  = s.gt & 31;
    const int     warp  = s.gt >> 5;
    const int     warps = s.G >> 5;
    const int     ldp   = s.nb + 1;
    for (int k = 0; k < n; k += s.nb)
    {
        const int w    = min(s.nb, n - k);
        const int R    = n - k;
        const int rest = R - w;
        // ---- the panel into shared memory
        for (int e = s.gt; e < R * w; e += s.G)
        {
            const int r = e / w, c = e - r * w;
            s.P[r * ldp + c] = s.f[(size_t)(k + r) * n + k + c];
        }
        for (int r = s.gt; r < R; r += s.G)
        {
            s.sigma[r] = r;
        }
        s.sync();
        // ---- factor it: per column a pivot search, the swap, the update
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
            K   pk = 0;
            int p  = INT_MAX;
            for (int q = 0; q < warps; ++q)
            {
                const K   kq = (K)s.red_key[q];
                const int rq = s.red_row[q];
                if (kq > pk || (kq == pk && rq < p))
                {
                    pk = kq;
                    p  = rq;
                }
            }
            if (p != jj)
            {
                for (int c = s.gt; c < w; c += s.G)
                {
                    const T t         = s.P[jj * ldp + c];
                    s.P[jj * ldp + c] = s.P[p * ldp + c];
                    s.P[p * ldp + c]  = t;
                }
            }
            if (s.gt == 0)
            {
                s.piv[k + jj] = k + p;
                const int t   = s.sigma[jj];
                s.sigma[jj]   = s.sigma[p];
                s.sigma[p]    = t;
            }
            s.sync();
            const T d = s.P[jj * ldp + jj];
            if (d == T(0))
            {
                if (s.gt == 0 && s.flags[0] < 0)
                {
                    s.flags[0] = k + jj;
                }
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
        // ---- the panel back; its interchanges as one permutation list
        for (int e = s.gt; e < R * w; e += s.G)
        {
            const int r = e / w, c = e - r * w;
            s.f[(size_t)(k + r) * n + k + c] = s.P[r * ldp + c];
        }
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
                    const int q            = cnt + __popc(bits & ((1u << lane) - 1u));
                    s.list[q]              = r;           // destination
                    s.list[2 * s.nb + q]   = s.sigma[r];  // source
                }
                cnt += __popc(bits);
            }
            if (lane == 0)
            {
                s.flags[1] = cnt;
            }
        }
        s.sync();
        const int cnt = s.flags[1];
        if (cnt > 0)
        {
            apply_interchanges(s, k, cnt, 0, k);
            apply_interchanges(s, k, cnt, k + w, n);
        }
        if (rest <= 0)
        {
            break;
        }
        // ---- U12 = L11^-1 A12 (thread per column) and L21 transposed
        for (int c = s.gt; c < rest; c += s.G)
        {
            T u[BatchTraits<T>::kMaxNB];
#pragma unroll
            for (int i = 0; i < BatchTraits<T>::kMaxNB; ++i)
            {
                u[i] = i < w ? s.f[(size_t)(k + i) * n + k + w + c] : T(0);
            }
#pragma unroll
            for (int i = 1; i < BatchTraits<T>::kMaxNB; ++i)
            {
                if (i < w)
                {
#pragma unroll
                    for (int j = 0; j < i; ++j)
                    {
                        u[i] = fma(-s.P[i * ldp + j], u[j], u[i]);
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < BatchTraits<T>::kMaxNB; ++i)
            {
                if (i < w)
                {
                    s.f[(size_t)(k + i) * n + k + w + c] = u[i];
                    s.U[i * s.np + c]                    = u[i];
                }
            }
        }
        for (int e = s.gt; e < rest * w; e += s.G)
        {
            const int r = e / w, c = e - r * w;
            s.LT[c * s.np + r] = s.P[(w + r) * ldp + c];
        }
        s.sync();
        // ---- A22 -= L21 U12: TM x TN tiles per thread, (G/16 TM) x (16 TN) per pass
        const int tx = s.gt & 15, ty = s.gt >> 4;
        const int th = (s.G >> 4) * TM, tw = 16 * TN;
        T*        c22 = s.f + (size_t)(k + w) * n + k + w;
        for (int i0 = 0; i0 < rest; i0 += th)
        {
            for (int j0 = 0; j0 < rest; j0 += tw)
            {
                const int ri = i0 + ty * TM, cj = j0 + tx * TN;
                if (ri < rest && cj < rest)
                {
                    T acc[TM][TN];
#pragma unroll
                    for (int a = 0; a < TM; ++a)
#pragma unroll
                        for (int b = 0; b < TN; ++b)
                            acc[a][b] = T(0);
                    for (int kk = 0; kk < w; ++kk)
                    {
                        T lv[TM], uv[TN];
#pragma unroll
                        for (int a = 0; a < TM; ++a)
                            lv[a] = s.LT[kk * s.np + ri + a];
#pragma unroll
                        for (int b = 0; b < TN; ++b)
                            uv[b] = s.U[kk * s.np + cj + b];
#pragma unroll
                        for (int a = 0; a < TM; ++a)
#pragma unroll
                            for (int b = 0; b < TN; ++b)
                                acc[a][b] = fma(lv[a], uv[b], acc[a][b]);
                    }
#pragma unroll
                    for (int a = 0; a < TM; ++a)
                    {
                        if (ri + a < rest)
                        {
                            T* crow = c22 + (size_t)(ri + a) * n + cj;
#pragma unroll
                            for (int b = 0; b < TN; ++b)
                            {
                                if (cj + b < rest)
                                {
                                    crow[b] -= acc[a][b];
                                }
                            }
                        }
                    }
                }
            }
        }
        s.sync();
    }
}

template <typename T>
__device__ void solve_system(Sys<T>& s, const double* __restrict__ a, const double* __restrict__ b,
    double* __restrict__ x, int max_iter, double tol, bool fallback, int32_t* status, double* berr, int sys)
{
    const int n    = s.n;
    const int lane = s.gt & 31, warp = s.gt >> 5;
    const int warps = s.G >> 5;
    if (s.gt == 0)
    {
        s.flags[0] = -1;
    }
    // ---- A -> F in T, ||A||_inf (a warp per row); the norm lands in r[0..)
    double anorm = 0.0;
    for (int i = warp; i < n; i += warps)
    {
        double acc = 0.0;
        for (int j = lane; j < n; j += 32)
        {
            const double v         = a[(size_t)i * n + j];
            s.f[(size_t)i * n + j] = (T)v;
            acc += fabs(v);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
        {
            acc += __shfl_down_sync(0xffffffffu, acc, off);
        }
        anorm = fmax(anorm, acc);
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
    // row permutation of the pivot sequence (n <= 512 swaps, one thread)
    if (s.gt == 0)
    {
        for (int i = 0; i < n; ++i)
        {
            s.perm[i] = i;
        }
        for (int i = 0; i < n; ++i)
        {
            const int t = s.piv[i];
            const int v = s.perm[i];
            s.perm[i]   = s.perm[t];
            s.perm[t]   = v;
        }
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
        for (int i = s.gt; i < n; i += s.G)
        {
            s.y[i] = s.r[s.perm[i]];
        }
        s.sync();
        bat_trsv(s, false);
        bat_trsv(s, true);
        for (int i = s.gt; i < n; i += s.G)
        {
            s.x[i] += s.y[i];
        }
        s.sync();
        // r = b - A x (a warp per row), max|r|, max|x|
        double rmax = 0.0, xmax = 0.0;
        for (int i = warp; i < n; i += warps)
        {
            double acc = 0.0;
            for (int j = lane; j < n; j += 32)
            {
                acc = fma(a[(size_t)i * n + j], s.x[j], acc);
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1)
            {
                acc += __shfl_down_sync(0xffffffffu, acc, off);
            }
            if (lane == 0)
            {
                const double ri = b[i] - acc;  // lane 0 holds the row's full sum
                s.r[i]          = ri;
                rmax            = fmax(rmax, fabs(ri));
                xmax            = fmax(xmax, fabs(s.x[i]));
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
                nb             = nb < 1 ? 1 : (nb > BatchTraits<T>::kMaxNB ? BatchTraits<T>::kMaxNB : nb);
                s_sys[0]       = sys0;
                bool fits      = true;
                for (int g = 1; g < kBT / G; ++g)
                {
                    const int q = atomicAdd(queue, 1);
                    s_sys[g]    = q < count ? (order != nullptr ? order[q] : q) : -1;
                    if (s_sys[g] >= 0 &&
                        group_layout<T>(sizes[s_sys[g]], nb).end > kBatchedSmem / (kBT / G) / 16 * 16)
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
                s.f                  = F + offa[sys];
                s.np                 = group_np(s.n);
                const GroupSmem L    = group_layout<T>(s.n, s.nb);
                unsigned char*  base = smem_raw + (size_t)group * (kBatchedSmem / (kBT / G) / 16 * 16);
                s.P                  = reinterpret_cast<T*>(base + L.P);
                s.LT                 = reinterpret_cast<T*>(base + L.LT);
                s.U                  = reinterpret_cast<T*>(base + L.U);
                s.y                  = reinterpret_cast<double*>(base + L.y);
                s.r                  = reinterpret_cast<double*>(base + L.r);
                s.x                  = reinterpret_cast<double*>(base + L.x);
                s.sigma              = reinterpret_cast<int*>(base + L.sigma);
                s.list               = reinterpret_cast<int*>(base + L.list);
                s.piv                = reinterpret_cast<int*>(base + L.piv);
                s.perm               = reinterpret_cast<int*>(base + L.perm);
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

// Whether the largest order of every bucket fits its group's shared-memory
// slice with the bucket's panel width (the systems are taken largest first,
// so a group never gets a larger one than its chunk's first).
template <typename T> bool table_fits(const int32_t* table_host)
{
    for (int bk = 0; bk < kBBuckets; ++bk)
    {
        const int e  = table_host[bk];
        const int G  = entry_g(e);
        const int nb = entry_nb(e);
        if (nb < 1 || nb > BatchTraits<T>::kMaxNB)
            return false;
        const int nmax = bk == kBBuckets - 1 ? kBMaxN : 64 * (bk + 1);
        if (group_layout<T>(nmax, nb).end > kBatchedSmem / (kBT / G) / 16 * 16)
            return false;
    }
    return true;
}
}  // namespace
int require_sm100();
}  // namespace b200la

using namespace b200la;

extern "C" {

B200LA_API size_t b200la_dgesv_batched_workspace_size(int64_t total_a, int64_t total_v, int precision)
{
    (void)total_v;
    (void)precision;
    if (total_a <= 0 || total_v <= 0)
        return 0;
    Arena a;
    a.next<int32_t>(64);  // queue counters of the two passes
    // factors: FP32 in the first pass; the FP64 pass for systems whose FP32
    // refinement stalled reuses the same buffer as FP64
    a.next<double>((size_t)total_a);
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
    const size_t need = b200la_dgesv_batched_workspace_size(total_a, total_v, precision);
    if (workspace == nullptr || workspace_bytes < need)
        return set_error(B200LA_WORKSPACE_TOO_SMALL, "dgesv_batched: workspace too small (%zu < %zu)",
            workspace_bytes, need);
    int rc = require_sm100();
    if (rc != B200LA_SUCCESS)
        return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Arena        ar(workspace, workspace_bytes);
    int32_t*     queue = ar.next<int32_t>(64);
    const int grid = device_sm_count();
    B200LA_CUDA(cudaMemsetAsync(queue, 0, sizeof(int32_t) * 2, s));
    void* fbuf = ar.next<double>((size_t)total_a);
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
