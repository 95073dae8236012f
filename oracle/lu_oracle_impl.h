/*
 * Type-generic body of the CPU oracle (included twice by lu_oracle.c, once
 * with T=double / SUF=d and once with T=float / SUF=s).
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference's NATIVE
 * LU-solve path, used by tests/ and by bench.py's CPU-baseline leg as the
 * oracle.  The B200 library never links, loads or calls it.
 *
 * Rounding is pinned to the reference build's: the reference's scalar loops
 * `y -= a * x` and `s += a * b` are contracted by g++ into single fused
 * multiply-adds, so every such update here is an explicit fma().  With that,
 * the factors, pivots and solutions below are bit-identical to the
 * reference's oracle/_ref build (checked by tests/test_oracle.py).
 */

#define OR_CAT2(a, b) a##b
#define OR_CAT(a, b) OR_CAT2(a, b)
#define OR_FN(name) OR_CAT(or_, OR_CAT(SUF, name))
#define OR_FMA OR_CAT(fma, FMA_SUF)
#define OR_ABS OR_CAT(fabs, FMA_SUF)

/* Panel width of the blocked LU, lu_decomposition_native.cpp:285
 * (kLuBlockSize = 64). */
#define OR_LU_BLOCK 64
/* Row-block height of the triangular solver, triangular_solver_native.cpp:17
 * (triangular_block = 32). */
#define OR_TRSM_BLOCK 32

/* y[c] -= a * x[c], c in [0, len): lu_decomposition_native.cpp:69-122
 * (lu_axpy_sub, scalar branch), one fused multiply-add per element. */
static void OR_CAT(axpy_sub_, SUF)(T* y, const T* x, T a, int64_t len)
{
    for (int64_t c = 0; c < len; ++c)
    {
        y[c] = OR_FMA(-a, x[c], y[c]);
    }
}

/* Row dot product, linear_solver_native.cpp:41-88 (lu_dot, scalar branch):
 * a single accumulator summed in index order.  The reference build (g++ -O3,
 * AVX2+FMA) computes that loop's products a full vector (4 doubles / 8
 * floats) at a time, then one half vector, and adds them one by one in
 * order, so those products are rounded before the add; the few products left
 * after that are fused into the sum.  The same rounding is reproduced here so
 * the solutions match the reference build bit for bit. */
static T OR_CAT(dots_, SUF)(const T* a, int64_t sa, const T* b, int64_t sb, int64_t count)
{
    const int64_t vec  = (int64_t)(32 / sizeof(T));
    const int64_t half = vec / 2;
    const int64_t main = count >= vec ? (count / vec) * vec : 0;
    T             s    = 0;
    int64_t       j    = 0;
    for (; j < main; ++j)
    {
        const T p = a[j * sa] * b[j * sb];
        s         = s + p;
    }
    if (count - j >= half)
    {
        for (int64_t q = 0; q < half; ++q, ++j)
        {
            const T p = a[j * sa] * b[j * sb];
            s         = s + p;
        }
    }
    for (; j < count; ++j)
    {
        s = OR_FMA(a[j * sa], b[j * sb], s);
    }
    return s;
}

static T OR_CAT(dot_, SUF)(const T* a, const T* b, int64_t count)
{
    return OR_CAT(dots_, SUF)(a, 1, b, 1, count);
}

/* The Cholesky pivot's reduction, dot(a_i, a_i, i) in
 * cholesky_decomposition_scalar_impl (both operands the same row): the
 * reference build compiles this inlined call of cholesky_dot differently from
 * its other call sites.  For double: whole vectors of 4 products rounded and
 * added in order, then the remaining (up to 3) products fused, with no half
 * vector; for float: as dots_.  Established by probing the reference build
 * with inputs that isolate one dot product of each call site and length. */
static T OR_CAT(dot_pivot_, SUF)(const T* a, int64_t count)
{
    if (sizeof(T) != 8)
    {
        return OR_CAT(dots_, SUF)(a, 1, a, 1, count);
    }
    const int64_t main = (count / 4) * 4;
    T             s    = 0;
    int64_t       j    = 0;
    for (; j < main; ++j)
    {
        const T p = a[j] * a[j];
        s         = s + p;
    }
    for (; j < count; ++j)
    {
        s = OR_FMA(a[j], a[j], s);
    }
    return s;
}

/* Unblocked panel factorization over columns [start, start+width), all rows
 * below: lu_decomposition_native.cpp:158-232 (lu_panel_factor).
 *  - pivot search: initial candidate |a[i][i]|, then rows i+1..n-1 with a
 *    strict '>' (first maximum wins; a NaN never displaces);
 *  - row swap over columns [0, start+width) only;
 *  - exactly-zero pivot: record the first one, skip the column;
 *  - multiplier: times 1/diag when |diag| >= smallest normal, else divided. */
static void OR_CAT(panel_, SUF)(T* m, int64_t n, int64_t start, int64_t width, int64_t* pivot,
    int64_t* first_zero)
{
    for (int64_t ii = 0; ii < width; ++ii)
    {
        const int64_t i   = start + ii;
        T*            row = m + i * n;
        T             mx  = OR_ABS(row[i]);
        int64_t       imx = i;
        for (int64_t k = i + 1; k < n; ++k)
        {
            const T v = OR_ABS(m[k * n + i]);
            if (v > mx)
            {
                mx  = v;
                imx = k;
            }
        }
        pivot[i] = imx + 1;
        if (imx != i)
        {
            T* prow = m + imx * n;
            for (int64_t j = 0; j < start + width; ++j)
            {
                const T t = row[j];
                row[j]    = prow[j];
                prow[j]   = t;
            }
        }
        const T diag = row[i];
        if (diag == (T)0)
        {
            if (*first_zero < 0)
            {
                *first_zero = i;
            }
            continue;
        }
        const int use_recip = OR_ABS(diag) >= T_MIN_NORMAL;
        const T   recip     = use_recip ? (T)((T)1 / diag) : (T)1;
        const T*  li        = row + start;
        for (int64_t r = i + 1; r < n; ++r)
        {
            T* lr = m + r * n + start;
            if (use_recip)
            {
                lr[ii] = lr[ii] * recip;
            }
            else
            {
                lr[ii] = lr[ii] / diag;
            }
            OR_CAT(axpy_sub_, SUF)(lr + ii + 1, li + ii + 1, lr[ii], width - ii - 1);
        }
    }
}

/* Replays pivot[start..start+width) on columns [start+width, n) in increasing
 * order: lu_decomposition_native.cpp:247-271 (lu_apply_pivots_to_trailing). */
static void OR_CAT(laswp_trailing_, SUF)(T* m, int64_t n, int64_t start, int64_t width,
    const int64_t* pivot)
{
    for (int64_t i = start; i < start + width; ++i)
    {
        const int64_t p = pivot[i] - 1;
        if (p != i)
        {
            T* ri = m + i * n;
            T* rp = m + p * n;
            for (int64_t j = start + width; j < n; ++j)
            {
                const T t = ri[j];
                ri[j]     = rp[j];
                rp[j]     = t;
            }
        }
    }
}

/* In-place blocked right-looking LU with partial pivoting of the row-major
 * n x n matrix m: lu_decomposition_native.cpp:329-429
 * (lu_decomposition_blocked_impl).  `delta` is rest*rest scratch (NULL lets
 * the oracle allocate it).  Returns 0 if U is nonsingular, else the 1-based
 * index of the first exactly-zero pivot (also written to *info). */
int OR_FN(getrf)(T* m, int64_t n, int64_t* pivot, int* info)
{
    if (m == NULL || pivot == NULL || n <= 0)
    {
        return -1;
    }
    for (int64_t i = 0; i < n; ++i)
    {
        pivot[i] = i + 1;
    }
    const int64_t rest0 = n > OR_LU_BLOCK ? n - OR_LU_BLOCK : 0;
    T*            delta = NULL;
    if (rest0 > 0)
    {
        delta = (T*)malloc(sizeof(T) * (size_t)rest0 * (size_t)rest0);
        if (delta == NULL)
        {
            return -2;
        }
    }
    int64_t first_zero = -1;
    for (int64_t k = 0; k < n; k += OR_LU_BLOCK)
    {
        const int64_t bs = (n - k) < OR_LU_BLOCK ? (n - k) : OR_LU_BLOCK;
        OR_CAT(panel_, SUF)(m, n, k, bs, pivot, &first_zero);
        const int64_t rest = n - k - bs;
        if (rest == 0)
        {
            continue;
        }
        OR_CAT(laswp_trailing_, SUF)(m, n, k, bs, pivot);
        /* U12 = L11^-1 A12 by row axpys, :370-380 */
        for (int64_t ii = 0; ii < bs; ++ii)
        {
            T* rowf = m + (k + ii) * n;
            T* ri   = rowf + k + bs;
            for (int64_t p = 0; p < ii; ++p)
            {
                OR_CAT(axpy_sub_, SUF)(ri, m + (k + p) * n + k + bs, rowf[k + p], rest);
            }
        }
        /* delta = L21 * U12 (multiplication_native.cpp:1701-1718, the
         * non-vectorized NN loop: c starts at 0, then c += a_ik * b_kj over k
         * in order), then A22 -= delta as a separate pass, :400-422. */
        for (int64_t r = 0; r < rest; ++r)
        {
            T*       dr = delta + r * rest;
            const T* lr = m + (k + bs + r) * n + k;
            for (int64_t c = 0; c < rest; ++c)
            {
                dr[c] = 0;
            }
            for (int64_t p = 0; p < bs; ++p)
            {
                const T  a  = lr[p];
                const T* up = m + (k + p) * n + k + bs;
                for (int64_t c = 0; c < rest; ++c)
                {
                    dr[c] = OR_FMA(a, up[c], dr[c]);
                }
            }
        }
        for (int64_t r = 0; r < rest; ++r)
        {
            OR_CAT(axpy_sub_, SUF)(m + (k + bs + r) * n + k + bs, delta + r * rest, (T)1, rest);
        }
    }
    free(delta);
    if (info)
    {
        *info = (int)(first_zero + 1);
    }
    return (int)(first_zero + 1);
}

/* Solve with existing factors, linear_solver_native.cpp:90-113 (lu_solve):
 * sequential pivot swaps on x, unit-lower forward substitution, then back
 * substitution dividing by U's diagonal. */
void OR_FN(getrs)(const T* m, const int64_t* pivot, int64_t n, T* x)
{
    for (int64_t i = 0; i < n; ++i)
    {
        const int64_t p = pivot[i] - 1;
        const T       t = x[i];
        x[i]            = x[p];
        x[p]            = t;
    }
    for (int64_t i = 0; i < n; ++i)
    {
        x[i] -= OR_CAT(dot_, SUF)(m + i * n, x, i);
    }
    for (int64_t i = n - 1; i >= 0; --i)
    {
        const T* ri = m + i * n;
        x[i]        = (x[i] - OR_CAT(dot_, SUF)(ri + i + 1, x + i + 1, n - i - 1)) / ri[i];
    }
}

int  OR_FN(potrf)(T* m, int64_t n, int upper, int* info);
void OR_FN(potrs)(const T* m, int64_t n, T* x);

/* linear_solver modes, linear_solver_native.cpp:149-191: mode 1 factors
 * then solves only if the factorization succeeded; mode 2 reuses the factors
 * and pivots; modes 3 and 4 are the Cholesky ones (factor lower, then
 * solve if positive definite; solve with the given factor).  Returns the
 * factorization status for modes 1 and 3, 0 for modes 2 and 4. */
int OR_FN(gesv)(T* m, int64_t* pivot, int64_t n, T* x, int mode)
{
    if (m == NULL || x == NULL || n <= 0)
    {
        return -1;
    }
    if (mode == 1)
    {
        const int st = OR_FN(getrf)(m, n, pivot, NULL);
        if (st == 0)
        {
            OR_FN(getrs)(m, pivot, n, x);
        }
        return st;
    }
    if (mode == 2)
    {
        OR_FN(getrs)(m, pivot, n, x);
        return 0;
    }
    if (mode == 3)
    {
        /* linear_solver_native.cpp: factor (lower), solve only if it succeeded */
        const int st = OR_FN(potrf)(m, n, 0, NULL);
        if (st == 0)
        {
            OR_FN(potrs)(m, n, x);
        }
        return st;
    }
    if (mode == 4)
    {
        OR_FN(potrs)(m, n, x);
        return 0;
    }
    return -1;
}

/* Inverse from a lower Cholesky factor, inversion_native.cpp:306-410
 * (cholesky_invert), three passes over the lower triangle of m:
 *  A. X = L^-1 in place, column j = 0..n-1 in order: x_jj = 1 / l_jj, then
 *     rows i = j+1..n-1 in order x_ij = -dot(m_i[j..i), x[j..i) of column j)
 *     / l_ii (row i right of column j and its diagonal still hold L);
 *  B. xt = X^T (only q >= p of xt_p written and read);
 *  C. a_ij for i <= j = dot(xt_i[j..n), xt_j[j..n)), then the lower
 *     triangle copied from the upper.
 * invert_dot (:147-204) is compiled without its vector branch in the
 * reference build; its loop rounds like dots_.  Returns -2 if the scratch
 * cannot be had. */
static int OR_CAT(chol_invert_, SUF)(T* m, int64_t n)
{
    T* col = (T*)malloc((size_t)n * sizeof(T));
    T* xt  = (T*)malloc((size_t)(n * n) * sizeof(T));
    if (col == NULL || xt == NULL)
    {
        free(col);
        free(xt);
        return -2;
    }
    for (int64_t j = 0; j < n; ++j)
    {
        const T d        = (T)1 / m[j * n + j];
        m[j * n + j] = d;
        col[j]           = d;
        for (int64_t i = j + 1; i < n; ++i)
        {
            T*      mi = m + i * n;
            const T v  = -OR_CAT(dot_, SUF)(mi + j, col + j, i - j) / mi[i];
            mi[j]      = v;
            col[i]     = v;
        }
    }
    for (int64_t p = 0; p < n; ++p)
    {
        for (int64_t q = p; q < n; ++q)
        {
            xt[p * n + q] = m[q * n + p];
        }
    }
    for (int64_t j = 0; j < n; ++j)
    {
        for (int64_t i = 0; i <= j; ++i)
        {
            m[i * n + j] = OR_CAT(dot_, SUF)(xt + i * n + j, xt + j * n + j, n - j);
        }
    }
    for (int64_t i = 1; i < n; ++i)
    {
        for (int64_t j = 0; j < i; ++j)
        {
            m[i * n + j] = m[j * n + i];
        }
    }
    free(col);
    free(xt);
    return 0;
}

/* Inverse from LU factors, inversion_native.cpp:228-304 (lu_invert):
 *  - inv = I, then rows (i, pivot[i]-1) swapped for i = 0..n-1 in order;
 *  - forward, rows i = 0..n-1: row_i -= m[i][k] row_k for k = 0..i-1 in
 *    order, one fused multiply-add per element (inv_axpy_sub, :82-126);
 *  - backward, rows i = n-1..0: row_i -= m[i][k] row_k for k = i+1..n-1 in
 *    order, then row_i *= 1 / m[i][i] (a reciprocal, then products);
 *  - m = inv.
 * Mode dispatch, inversion_native.cpp:412-452: mode 1 factors m first and
 * inverts only if the factorization found no exact zero pivot (m then keeps
 * the factors); mode 2 inverts the factors and pivots as given; mode 3
 * factors m (lower Cholesky) and inverts only if every pivot was positive
 * (m then keeps the partial factor); mode 4 inverts the lower factor given
 * in m (its upper triangle is not read).  Returns the getrf (potrf) status
 * for mode 1 (3), 0 for modes 2 and 4, -1 for invalid arguments. */
int OR_FN(getri)(T* m, int64_t* pivot, int64_t n, int mode)
{
    if (m == NULL || n <= 0 || mode < 1 || mode > 4 || (mode <= 2 && pivot == NULL))
    {
        return -1;
    }
    if (mode >= 3)
    {
        const int pst = mode == 3 ? OR_FN(potrf)(m, n, 0, NULL) : 0;
        if (pst != 0)
        {
            return pst;
        }
        return OR_CAT(chol_invert_, SUF)(m, n);
    }
    int st = 0;
    if (mode == 1)
    {
        st = OR_FN(getrf)(m, n, pivot, NULL);
        if (st != 0)
        {
            return st;
        }
    }
    T* inv = (T*)calloc((size_t)(n * n), sizeof(T));
    if (inv == NULL)
    {
        return -2;
    }
    for (int64_t i = 0; i < n; ++i)
    {
        inv[i * n + i] = (T)1;
    }
    for (int64_t i = 0; i < n; ++i)
    {
        const int64_t p = pivot[i] - 1;
        if (p != i)
        {
            for (int64_t c = 0; c < n; ++c)
            {
                const T t        = inv[i * n + c];
                inv[i * n + c] = inv[p * n + c];
                inv[p * n + c] = t;
            }
        }
    }
    for (int64_t i = 0; i < n; ++i)
    {
        for (int64_t k = 0; k < i; ++k)
        {
            OR_CAT(axpy_sub_, SUF)(inv + i * n, inv + k * n, m[i * n + k], n);
        }
    }
    for (int64_t i = n - 1; i >= 0; --i)
    {
        for (int64_t k = i + 1; k < n; ++k)
        {
            OR_CAT(axpy_sub_, SUF)(inv + i * n, inv + k * n, m[i * n + k], n);
        }
        const T inv_diag = (T)1 / m[i * n + i];
        for (int64_t c = 0; c < n; ++c)
        {
            inv[i * n + c] *= inv_diag;
        }
    }
    for (int64_t e = 0; e < n * n; ++e)
    {
        m[e] = inv[e];
    }
    free(inv);
    return st;
}

/* Determinant, determinant.cpp:18-37 (lu_determinant / cholesky_determinant:
 * the product of the factor's diagonal in index order, no pivot sign, not
 * squared for Cholesky) and :56-90 (modes): mode 1 factors m in place (LU)
 * and returns the product if the factorization found no exact zero pivot,
 * else 0; mode 3 likewise with the lower Cholesky factor (0 if m is not
 * positive definite); modes 2 and 4 multiply the diagonal of m as given.
 * *status: the factorization's status (modes 1, 3), 0 (modes 2, 4) or -1
 * (invalid). */
T OR_FN(det)(T* m, int64_t* pivot, int64_t n, int mode, int* status)
{
    *status = -1;
    if (m == NULL || n <= 0 || mode < 1 || mode > 4 || (mode == 1 && pivot == NULL))
    {
        return (T)0;
    }
    *status = 0;
    if (mode == 1 || mode == 3)
    {
        *status = mode == 1 ? OR_FN(getrf)(m, n, pivot, NULL) : OR_FN(potrf)(m, n, 0, NULL);
        if (*status != 0)
        {
            return (T)0;
        }
    }
    T det = m[0];
    for (int64_t i = 1; i < n; ++i)
    {
        det *= m[i * n + i];
    }
    return det;
}

/* Reduction `sum -= a[j] * b[j]` over j in order, as the reference build
 * compiles it (see dots_: full vectors of products rounded, then one half
 * vector, subtracted one by one in order; the rest fused). */
static T OR_CAT(dots_sub_, SUF)(T sum, const T* a, int64_t sa, const T* b, int64_t sb, int64_t count)
{
    const int64_t vec  = (int64_t)(32 / sizeof(T));
    const int64_t half = vec / 2;
    const int64_t main = count >= vec ? (count / vec) * vec : 0;
    int64_t       j    = 0;
    for (; j < main; ++j)
    {
        const T p = a[j * sa] * b[j * sb];
        sum       = sum - p;
    }
    if (count - j >= half)
    {
        for (int64_t q = 0; q < half; ++q, ++j)
        {
            const T p = a[j * sa] * b[j * sb];
            sum       = sum - p;
        }
    }
    for (; j < count; ++j)
    {
        sum = OR_FMA(-a[j * sa], b[j * sb], sum);
    }
    return sum;
}

/* Unblocked Cholesky of the n x n diagonal block at A (row stride lda):
 * cholesky_decomposition_native.cpp (cholesky_decomposition_scalar_impl),
 * row by row: a_ij = (a_ij - dot(a_i, a_j, j)) / a_jj for j < i (a_ji = 0),
 * then a_ii = sqrt(a_ii - dot(a_i, a_i, i)) (dot_pivot_'s rounding);
 * returns i + 1 at the first non-positive pivot, else 0. */
static int64_t OR_CAT(potf2_, SUF)(int64_t n, T* A, int64_t lda)
{
    for (int64_t i = 0; i < n; ++i)
    {
        T* ai = A + i * lda;
        for (int64_t j = 0; j < i; ++j)
        {
            T*      aj  = A + j * lda;
            const T sum = ai[j] - OR_CAT(dot_, SUF)(ai, aj, j);
            ai[j]       = sum / aj[j];
            aj[i]       = (T)0;
        }
        const T sum = ai[i] - OR_CAT(dot_pivot_, SUF)(ai, i);
        if (sum <= (T)0)
        {
            return i + 1;
        }
        ai[i] = (T)sqrt((double)sum);
    }
    return 0;
}

/* Blocked lower Cholesky of the row-major n x n matrix m (lda = n):
 * cholesky_decomposition_native.cpp (cholesky_decomposition_blocked_lower,
 * block 64, the non-vectorized trailing update): per block, the diagonal
 * block by potf2, zeros right of it in its rows, A21 = A21 L11^-T row by row
 * (row[j] = (row[j] - dot(row, l_j, j)) / l_jj), then for the trailing
 * lower triangle t_ij -= dot(a21_i, a21_j, bs).  upper != 0: the factor is
 * transposed into the upper triangle and the lower one cleared
 * (cholesky_decomposition_apply_impl).  Returns 0, or the 1-based index of
 * the first non-positive pivot (*info too). */
int OR_FN(potrf)(T* m, int64_t n, int upper, int* info)
{
    if (m == NULL || n <= 0)
    {
        return -1;
    }
    int64_t rc = 0;
    for (int64_t k = 0; k < n && rc == 0; k += 64)
    {
        const int64_t bs  = (n - k) < 64 ? (n - k) : 64;
        T*            l11 = m + k * n + k;
        const int64_t r   = OR_CAT(potf2_, SUF)(bs, l11, n);
        if (r != 0)
        {
            rc = k + r;
            break;
        }
        for (int64_t i = k; i < k + bs; ++i)
        {
            for (int64_t j = k + bs; j < n; ++j)
            {
                m[i * n + j] = (T)0;
            }
        }
        const int64_t below = n - k - bs;
        if (below == 0)
        {
            continue;
        }
        T* a21 = m + (k + bs) * n + k;
        T* a22 = m + (k + bs) * n + k + bs;
        for (int64_t r2 = 0; r2 < below; ++r2)
        {
            T* row = a21 + r2 * n;
            for (int64_t j = 0; j < bs; ++j)
            {
                const T* lj  = l11 + j * n;
                const T  sum = row[j] - OR_CAT(dot_, SUF)(row, lj, j);
                row[j]       = sum / lj[j];
            }
        }
        for (int64_t i = 0; i < below; ++i)
        {
            for (int64_t j = 0; j <= i; ++j)
            {
                a22[i * n + j] -= OR_CAT(dot_, SUF)(a21 + i * n, a21 + j * n, bs);
            }
        }
    }
    if (rc == 0 && upper)
    {
        for (int64_t i = 0; i < n; ++i)
        {
            for (int64_t j = 0; j < i; ++j)
            {
                m[j * n + i] = m[i * n + j];
                m[i * n + j] = (T)0;
            }
        }
    }
    if (info)
    {
        *info = (int)rc;
    }
    return (int)rc;
}

/* Solve with a lower Cholesky factor: linear_solver_native.cpp
 * (cholesky_solve): forward x_i = (x_i - sum_{j<i} l_ij x_j) / l_ii, then
 * backward x_i = (x_i - sum_{j>i} l_ji x_j) / l_ii reading the factor's
 * column i; both reductions round as the reference build compiles them
 * (dots_sub_; the backward one's loads are strided, the rounding the same). */
void OR_FN(potrs)(const T* m, int64_t n, T* x)
{
    for (int64_t i = 0; i < n; ++i)
    {
        const T* ri  = m + i * n;
        const T  sum = OR_CAT(dots_sub_, SUF)(x[i], ri, 1, x, 1, i);
        x[i]         = sum / ri[i];
    }
    for (int64_t i = n - 1; i >= 0; --i)
    {
        const T sum = OR_CAT(dots_sub_, SUF)(x[i], m + (i + 1) * n + i, n, x + i + 1, 1, n - i - 1);
        x[i]        = sum / m[i * n + i];
    }
}

/* transpose::apply, transpose_native.cpp: the row-major rows x cols matrix
 * m becomes its row-major cols x rows transpose in place.  Square: the
 * reference swaps m[i][j] and m[j][i] (j > i) tile by tile; otherwise it
 * follows the permutation cycles of the in-place transposition.  Both are
 * data movement, so this restatement swaps the square case and transposes
 * the other through scratch (rows*cols elements) and copies back: the same
 * result.  Returns -1 for invalid arguments. */
int OR_FN(transpose)(int64_t rows, int64_t cols, T* m, T* scratch)
{
    if (!m || rows <= 0 || cols <= 0 || (rows != cols && !scratch))
    {
        return -1;
    }
    if (rows == cols)
    {
        for (int64_t i = 0; i < rows; ++i)
        {
            for (int64_t j = i + 1; j < rows; ++j)
            {
                const T t        = m[i * rows + j];
                m[i * rows + j]  = m[j * rows + i];
                m[j * rows + i]  = t;
            }
        }
        return 0;
    }
    for (int64_t i = 0; i < rows; ++i)
    {
        for (int64_t j = 0; j < cols; ++j)
        {
            scratch[j * rows + i] = m[i * cols + j];
        }
    }
    for (int64_t e = 0; e < rows * cols; ++e)
    {
        m[e] = scratch[e];
    }
    return 0;
}

/* Batched product c_i = a_i b_i of `count` packed dim x dim matrices:
 * multiplication_batched_cublas.cu:15-40 (batched_matmul_kernel: each entry
 * sum += a b from zero in k order, which nvcc contracts into fused
 * multiply-adds).  The reference has no CPU version. */
int OR_FN(gemm_batched)(int64_t dim, int64_t count, const T* a, const T* b, T* c)
{
    if (!a || !b || !c || dim <= 0 || count <= 0)
    {
        return -1;
    }
    const int64_t ms = dim * dim;
    for (int64_t q = 0; q < count; ++q)
    {
        const T* A  = a + q * ms;
        const T* B  = b + q * ms;
        T*       Cq = c + q * ms;
        for (int64_t r = 0; r < dim; ++r)
        {
            for (int64_t j = 0; j < dim; ++j)
            {
                T sum = (T)0;
                for (int64_t k = 0; k < dim; ++k)
                {
                    sum = OR_FMA(A[r * dim + k], B[k * dim + j], sum);
                }
                Cq[r * dim + j] = sum;
            }
        }
    }
    return 0;
}

/* c = alpha op(a) op(b) + beta c, row-major, BLAS contract:
 * multiplication_native.cpp:1542-1567 (beta applied up front; beta == 0
 * overwrites c), :1807-1814 (alpha == 0 quick return), and the scalar loop
 * nests :1701-1787 for the four transpose combinations. */
int OR_FN(gemm)(int ta, int tb, int64_t rows, int64_t cols, int64_t depth, T alpha, const T* a,
    int64_t lda, const T* b, int64_t ldb, T beta, T* c, int64_t ldc)
{
    if (!a || !b || !c || rows <= 0 || cols <= 0 || depth <= 0 || lda <= 0 || ldb <= 0 || ldc <= 0)
    {
        return -1;
    }
    if (beta != (T)1)
    {
        for (int64_t i = 0; i < rows; ++i)
        {
            for (int64_t j = 0; j < cols; ++j)
            {
                c[i * ldc + j] = beta == (T)0 ? (T)0 : c[i * ldc + j] * beta;
            }
        }
    }
    if (alpha == (T)0)
    {
        return 0;
    }
    if (!ta && !tb)
    {
        for (int64_t i = 0; i < rows; ++i)
        {
            for (int64_t k = 0; k < depth; ++k)
            {
                const T s = alpha * a[i * lda + k];
                for (int64_t j = 0; j < cols; ++j)
                {
                    c[i * ldc + j] = OR_FMA(s, b[k * ldb + j], c[i * ldc + j]);
                }
            }
        }
    }
    else if (ta && !tb)
    {
        for (int64_t k = 0; k < depth; ++k)
        {
            for (int64_t i = 0; i < rows; ++i)
            {
                const T s = alpha * a[k * lda + i];
                for (int64_t j = 0; j < cols; ++j)
                {
                    c[i * ldc + j] = OR_FMA(s, b[k * ldb + j], c[i * ldc + j]);
                }
            }
        }
    }
    else
    {
        for (int64_t i = 0; i < rows; ++i)
        {
            for (int64_t j = 0; j < cols; ++j)
            {
                /* the reference's dot loops (contiguous for NT, strided a
                 * for TT) round like lu_dot in its build */
                const T s = ta ? OR_CAT(dots_, SUF)(a + i, lda, b + j * ldb, 1, depth)
                               : OR_CAT(dot_, SUF)(a + i * lda, b + j * ldb, depth);
                c[i * ldc + j] = OR_FMA(alpha, s, c[i * ldc + j]);
            }
        }
    }
    return 0;
}

/* op(A) X = B, triangular_solver_native.cpp:67-179: X = B, then row blocks of
 * 32 in substitution order; inside a block, sequential row axpys and a
 * division by the diagonal (unless unit); below/above it, a GEMM of the
 * solved block followed by a separate subtraction pass.  A and B are only
 * read, only the selected triangle is read, the diagonal is not read when
 * unit != 0.  Argument checks as src/common/triangular_solver_checks.h:11-35. */
int OR_FN(trsm)(int upper, int transpose, int unit, int64_t n, int64_t nrhs, const T* a,
    int64_t lda, const T* b, int64_t ldb, T* x, int64_t ldx)
{
    if (n <= 0 || nrhs <= 0 || n > 2147483647LL || nrhs > 2147483647LL)
    {
        return -1;
    }
    if (!a || !b || !x || a == b || a == x || b == x)
    {
        return -1;
    }
    if (lda < n || ldb < nrhs || ldx < nrhs)
    {
        return -1;
    }
    const int64_t lim = INT64_MAX / n;
    if (lda > lim || ldb > lim || ldx > lim)
    {
        return -1;
    }
    T* update = NULL;
    if (n > OR_TRSM_BLOCK)
    {
        update = (T*)malloc(sizeof(T) * (size_t)n * (size_t)nrhs);
        if (!update)
        {
            return -2;
        }
    }
    for (int64_t i = 0; i < n; ++i)
    {
        for (int64_t j = 0; j < nrhs; ++j)
        {
            x[i * ldx + j] = b[i * ldb + j];
        }
    }
#define OR_COEF(i, j) (transpose ? a[(j) * lda + (i)] : a[(i) * lda + (j)])
    const int eff_upper = (upper != 0) != (transpose != 0);
    for (int64_t done = 0; done < n; done += OR_TRSM_BLOCK)
    {
        const int64_t width = (n - done) < OR_TRSM_BLOCK ? (n - done) : OR_TRSM_BLOCK;
        const int64_t begin = eff_upper ? n - done - width : done;
        const int64_t end   = begin + width;
        for (int64_t step = 0; step < width; ++step)
        {
            const int64_t i   = eff_upper ? end - step - 1 : begin + step;
            T*            row = x + i * ldx;
            const int64_t k0  = eff_upper ? i + 1 : begin;
            const int64_t k1  = eff_upper ? end : i;
            for (int64_t k = k0; k < k1; ++k)
            {
                OR_CAT(axpy_sub_, SUF)(row, x + k * ldx, OR_COEF(i, k), nrhs);
            }
            if (!unit)
            {
                const T d = OR_COEF(i, i);
                for (int64_t j = 0; j < nrhs; ++j)
                {
                    row[j] = row[j] / d;
                }
            }
        }
        const int64_t first = eff_upper ? 0 : end;
        const int64_t rows  = eff_upper ? begin : n - end;
        if (rows == 0)
        {
            continue;
        }
        const T* blk = transpose ? a + begin * lda + first : a + first * lda + begin;
        OR_FN(gemm)(transpose, 0, rows, nrhs, width, (T)1, blk, lda, x + begin * ldx, ldx, (T)0,
            update, nrhs);
        for (int64_t r = 0; r < rows; ++r)
        {
            OR_CAT(axpy_sub_, SUF)(x + (first + r) * ldx, update + r * nrhs, (T)1, nrhs);
        }
    }
#undef OR_COEF
    free(update);
    return 0;
}

#undef OR_CAT2
#undef OR_CAT
#undef OR_FN
#undef OR_FMA
#undef OR_ABS
#undef OR_LU_BLOCK
#undef OR_TRSM_BLOCK
