/*
 * CPU oracle for the LU-solve path: a plain-C restatement of the reference's
 * NATIVE algorithm (see lu_oracle_impl.h for the per-function citations).
 *
 * TEST INFRASTRUCTURE ONLY.  Imported by tests/, by __graft_entry__.smoke()
 * and by bench.py's CPU-baseline leg as the oracle; the B200 library never
 * links or calls it.  Parity is pinned two ways: bit-for-bit against the
 * reference's own sources compiled into oracle/_ref (oracle/Makefile), and
 * against the committed fixtures in tests/golden/ that were produced by that
 * reference build.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#define T double
#define SUF d
#define FMA_SUF
#define T_MIN_NORMAL DBL_MIN
#include "lu_oracle_impl.h"
#undef T
#undef SUF
#undef FMA_SUF
#undef T_MIN_NORMAL

#define T float
#define SUF s
#define FMA_SUF f
#define T_MIN_NORMAL FLT_MIN
#include "lu_oracle_impl.h"
#undef T
#undef SUF
#undef FMA_SUF
#undef T_MIN_NORMAL

/* Normwise backward error of x for A x = b (infinity norms):
 *   eta = ||b - A x|| / (||A|| ||x|| + ||b||),
 * with the residual accumulated in long double.  Used by the tests as the
 * accuracy metric the path is held to. */
double or_backward_error(const double* a, int64_t n, int64_t lda, const double* x,
    const double* b)
{
    long double rmax = 0, anorm = 0, xmax = 0, bmax = 0;
    for (int64_t i = 0; i < n; ++i)
    {
        long double s = b[i], rs = 0;
        for (int64_t j = 0; j < n; ++j)
        {
            s -= (long double)a[i * lda + j] * (long double)x[j];
            rs += fabsl((long double)a[i * lda + j]);
        }
        if (fabsl(s) > rmax) rmax = fabsl(s);
        if (rs > anorm) anorm = rs;
        if (fabsl((long double)x[i]) > xmax) xmax = fabsl((long double)x[i]);
        if (fabsl((long double)b[i]) > bmax) bmax = fabsl((long double)b[i]);
    }
    const long double den = anorm * xmax + bmax;
    return den > 0 ? (double)(rmax / den) : 0.0;
}

/* Smallest relative gap between the winning and the runner-up |candidate| of
 * every pivot search of the oracle's own factorization of a copy of m: the
 * "near-tie" measure used to reject inputs whose pivot order could flip under
 * a different (but equally valid) rounding order. */
double or_dmin_pivot_gap(const double* m_in, int64_t n)
{
    double* m = (double*)malloc(sizeof(double) * (size_t)n * (size_t)n);
    int64_t* piv = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
    double gap = INFINITY;
    if (!m || !piv) { free(m); free(piv); return -1.0; }
    for (int64_t i = 0; i < n * n; ++i) m[i] = m_in[i];
    /* Unblocked elimination with the same pivot rule; only the gap matters,
     * so the rounding order of the updates is irrelevant here. */
    for (int64_t i = 0; i < n; ++i)
    {
        double best = -1, second = -1; int64_t bi = i;
        for (int64_t k = i; k < n; ++k)
        {
            const double v = fabs(m[k * n + i]);
            if (v > best) { second = best; best = v; bi = k; }
            else if (v > second) second = v;
        }
        if (best > 0 && second >= 0 && n - i > 1)
        {
            const double g = (best - second) / best;
            if (g < gap) gap = g;
        }
        if (bi != i)
            for (int64_t j = 0; j < n; ++j) { double t = m[i*n+j]; m[i*n+j] = m[bi*n+j]; m[bi*n+j] = t; }
        const double d = m[i * n + i];
        if (d == 0) continue;
        for (int64_t r = i + 1; r < n; ++r)
        {
            const double l = m[r * n + i] / d;
            m[r * n + i] = l;
            for (int64_t j = i + 1; j < n; ++j) m[r * n + j] -= l * m[i * n + j];
        }
    }
    free(m); free(piv);
    return gap;
}
