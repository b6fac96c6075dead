/*
 * oracle.c -- CPU restatement of the reference's factor-and-solve arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the parity tests, the smoke check
 * and the benchmark's CPU-baseline leg compare the CUDA library against.  The library
 * (libops_solver.so) never links, loads or calls it.
 *
 * Each routine restates one reference kernel's per-element operation order so that the
 * CUDA kernels can be checked bit for bit (paths relative to the reference project root):
 *   orc_spotrf_simt     src/cholesky/arch35/cholesky_simt.cpp:52-92        (n <= 8)
 *   orc_spotrf_group    src/cholesky/arch35/cholesky_vector.cpp:588-794    (9 <= n <= 32)
 *                       with StoreSmallCompleted :837-862 (failed slots keep unfinished columns)
 *   orc_spotrs_simt     src/cholesky/arch35/cholesky_simt.cpp:93-117       (SolveKernel)
 *   orc_spotrs_dot      src/cholesky/arch35/cholesky_vector.cpp:30-122     (VectorTriSolve, AccumulateDot)
 *   orc_sgetrf          src/utils/kernel/real_lu.hpp:59-139 (first-max pivot, NaN rule),
 *                       :216-311 (swap, IEEE division), :345-368 (FMA rank-1), :409-448 (loop, info)
 *   orc_sgetri_vector   src/sgetri/real_lu_blocked_inverse_kernel.cpp:676-830,1040-1044
 * Routines for sizes where the reference hands its arithmetic to a third-party Cube GEMM
 * (CATLASS / CANN MatmulImpl) restate this build's own order instead, and say so:
 *   orc_spotrf_fma      right-looking Cholesky with FMA updates in ascending k (33..256)
 *   orc_spotrf_blocked  the same in 64-column panels with panel partial sums (n > 256)
 *   orc_spotrs_right    right-looking Cholesky solve in 64-row blocks (n > 128)
 *   orc_sgetrs          column-oriented LU solve (math of test/utils/lu_verify_utils.py:67-192)
 *   orc_cpotrf/cpotrs   complex64 Cholesky factor and solve, FMA order (see their comment);
 *                       above order 240 in 64-column panels with panel partial sums
 *
 * Compiled with -ffp-contract=off: every fused multiply-add is an explicit fmaf().
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define FLT_MAX_VALUE 3.402823466e38F

/* Element (i, j) of the factor triangle: lower reads A[i + j*lda], upper reads the mirror
 * A[j + i*lda] (cholesky_simt.cpp:19-22, Offset). */
static inline int64_t tri_at(int lda, int upper, int i, int j)
{
    return upper ? (int64_t)i * lda + j : (int64_t)j * lda + i;
}

/* ---------------------------------------------------------------------------------------
 * Real Cholesky
 * ------------------------------------------------------------------------------------- */

/* n <= 8: left-looking dot products with fmaf, sqrt refined once by its FMA residual,
 * IEEE division of the column (cholesky_simt.cpp:64-90).  Returns info. */
int orc_spotrf_simt(int n, float *a, int lda, int upper)
{
    for (int k = 0; k < n; ++k)
    {
        float d = a[(int64_t)k * (lda + 1)];
        for (int t = 0; t < k; ++t)
        {
            float f = a[tri_at(lda, upper, k, t)];
            d = fmaf(-f, f, d);
        }
        if (!(d > 0)) return k + 1;
        float root = sqrtf(d);
        float correction = fmaf(-root, root, d);
        d = fmaf(correction, 0.5f / root, root);
        a[(int64_t)k * (lda + 1)] = d;
        for (int i = k + 1; i < n; ++i)
        {
            float x = a[tri_at(lda, upper, i, k)];
            for (int t = 0; t < k; ++t) x = fmaf(-a[tri_at(lda, upper, i, t)], a[tri_at(lda, upper, k, t)], x);
            a[tri_at(lda, upper, i, k)] = x / d;
        }
    }
    return 0;
}

/* 9 <= n <= 32 (any n is accepted): right-looking in groups of four columns.  Per column:
 * pivot check d > 0 && d <= FLT_MAX, IEEE sqrt, IEEE division of the rows below, the
 * diagonal stores sqrt(d) itself; in-group updates a -= (l * alpha) with separate rounding;
 * after the group, a rank-4 trailing update a -= (((p0 + p1) + p2) + p3), every product and
 * sum rounded separately (cholesky_vector.cpp:588-794).  A failed matrix keeps only its
 * completed columns (StoreSmallCompleted, :837-862): columns >= info-1 of the caller's
 * matrix are left as they were. */
int orc_spotrf_group(int n, float *a, int lda, int upper)
{
    /* Work on a private dense lower copy w[j*n + i] = A(i, j). */
    float *w = (float *)malloc(sizeof(float) * (size_t)n * (size_t)n + 4);
    for (int j = 0; j < n; ++j)
        for (int i = j; i < n; ++i) w[(size_t)j * n + i] = a[tri_at(lda, upper, i, j)];
    int failure = 0;
    for (int base = 0; base < n && !failure; base += 4)
    {
        int end = base + 4;
        for (int k = base; k < end && k < n; ++k)
        {
            float d = w[(size_t)k * n + k];
            if (!(d > 0.0f && d <= FLT_MAX_VALUE))
            {
                failure = k + 1;
                break;
            }
            float s = sqrtf(d);
            for (int i = k + 1; i < n; ++i) w[(size_t)k * n + i] = w[(size_t)k * n + i] / s;
            w[(size_t)k * n + k] = s;
            for (int j = k + 1; j < end && j < n; ++j)
            {
                float alpha = w[(size_t)k * n + j];
                for (int i = j; i < n; ++i)
                {
                    float product = w[(size_t)k * n + i] * alpha;
                    w[(size_t)j * n + i] = w[(size_t)j * n + i] - product;
                }
            }
        }
        if (failure) break;
        for (int j = end; j < n; ++j)
        {
            float a0 = w[(size_t)base * n + j], a1 = w[(size_t)(base + 1) * n + j];
            float a2 = w[(size_t)(base + 2) * n + j], a3 = w[(size_t)(base + 3) * n + j];
            for (int i = j; i < n; ++i)
            {
                float sum = w[(size_t)base * n + i] * a0;
                float p = w[(size_t)(base + 1) * n + i] * a1;
                sum = sum + p;
                p = w[(size_t)(base + 2) * n + i] * a2;
                sum = sum + p;
                p = w[(size_t)(base + 3) * n + i] * a3;
                sum = sum + p;
                w[(size_t)j * n + i] = w[(size_t)j * n + i] - sum;
            }
        }
    }
    int done = failure ? failure - 1 : n;
    for (int j = 0; j < done; ++j)
        for (int i = j; i < n; ++i) a[tri_at(lda, upper, i, j)] = w[(size_t)j * n + i];
    free(w);
    return failure;
}

/* n > 32 (this build's order; the reference uses a CATLASS FP32 Gram product here):
 * right-looking, IEEE sqrt and division, trailing updates a = fmaf(-l_ik, l_jk, a) applied
 * in ascending k.  Any blocking that keeps each element's ascending-k FMA sequence
 * reproduces these bits.  A failed matrix keeps only its completed columns. */
int orc_spotrf_fma(int n, float *a, int lda, int upper)
{
    float *w = (float *)malloc(sizeof(float) * (size_t)n * (size_t)n + 4);
    for (int j = 0; j < n; ++j)
        for (int i = j; i < n; ++i) w[(size_t)j * n + i] = a[tri_at(lda, upper, i, j)];
    int failure = 0;
    for (int k = 0; k < n; ++k)
    {
        float d = w[(size_t)k * n + k];
        if (!(d > 0.0f && d <= FLT_MAX_VALUE))
        {
            failure = k + 1;
            break;
        }
        float s = sqrtf(d);
        w[(size_t)k * n + k] = s;
        for (int i = k + 1; i < n; ++i) w[(size_t)k * n + i] = w[(size_t)k * n + i] / s;
        for (int j = k + 1; j < n; ++j)
        {
            float ljk = w[(size_t)k * n + j];
            for (int i = j; i < n; ++i) w[(size_t)j * n + i] = fmaf(-w[(size_t)k * n + i], ljk, w[(size_t)j * n + i]);
        }
    }
    int done = failure ? failure - 1 : n;
    for (int j = 0; j < done; ++j)
        for (int i = j; i < n; ++i) a[tri_at(lda, upper, i, j)] = w[(size_t)j * n + i];
    free(w);
    return failure;
}

/* Above order 256 (this build's order for the whole-GPU factorisation; the reference hands
 * these orders to a blocked Gram product): right-looking in panels of ORC_NB = 64 columns.
 * Inside a panel every element takes the panel's updates one by one, fmaf(-l_ik, l_jk, a_ij)
 * in ascending k, and each column is divided as it is finished; an element right of the
 * panel takes the panel's products as one partial sum t = fmaf(l_ik, l_jk, t) from zero in
 * ascending k, then a_ij - t.  The partial sums keep each element's chain of roundings at
 * n / 64 subtractions plus 64-term sums (the size of a blocked LAPACK's) instead of n, which
 * the reference's residual gate needs at orders in the thousands. */
#define ORC_NB 64
int orc_spotrf_blocked(int n, float *a, int lda, int upper)
{
    float *w = (float *)malloc(sizeof(float) * (size_t)n * (size_t)n + 4);
    for (int j = 0; j < n; ++j)
        for (int i = j; i < n; ++i) w[(size_t)j * n + i] = a[tri_at(lda, upper, i, j)];
    int failure = 0;
    for (int k0 = 0; k0 < n && !failure; k0 += ORC_NB)
    {
        const int kend = k0 + ORC_NB < n ? k0 + ORC_NB : n;
        for (int k = k0; k < kend; ++k)
        {
            float d = w[(size_t)k * n + k];
            if (!(d > 0.0f && d <= FLT_MAX_VALUE))
            {
                failure = k + 1;
                break;
            }
            float s = sqrtf(d);
            w[(size_t)k * n + k] = s;
            for (int i = k + 1; i < n; ++i) w[(size_t)k * n + i] = w[(size_t)k * n + i] / s;
            for (int j = k + 1; j < kend; ++j)
            {
                float ljk = w[(size_t)k * n + j];
                for (int i = j; i < n; ++i) w[(size_t)j * n + i] = fmaf(-w[(size_t)k * n + i], ljk, w[(size_t)j * n + i]);
            }
        }
        if (failure) break;
        for (int j = kend; j < n; ++j)
            for (int i = j; i < n; ++i)
            {
                float t = 0.0f;
                for (int k = k0; k < kend; ++k) t = fmaf(w[(size_t)k * n + i], w[(size_t)k * n + j], t);
                w[(size_t)j * n + i] = w[(size_t)j * n + i] - t;
            }
    }
    int done = failure ? failure - 1 : n;
    for (int j = 0; j < done; ++j)
        for (int i = j; i < n; ++i) a[tri_at(lda, upper, i, j)] = w[(size_t)j * n + i];
    free(w);
    return failure;
}

/* The size dispatch of SpotrfBatched / Spotrf in this build. */
int orc_spotrf(int n, float *a, int lda, int upper)
{
    if (n <= 8) return orc_spotrf_simt(n, a, lda, upper);
    if (n <= 32) return orc_spotrf_group(n, a, lda, upper);
    if (n <= 256) return orc_spotrf_fma(n, a, lda, upper);
    return orc_spotrf_blocked(n, a, lda, upper);
}

/* SolveKernel (cholesky_simt.cpp:93-117): per right-hand side a forward then a backward
 * substitution, each x = fmaf(-l, b_j, x) in ascending (forward) or ascending-from-i+1
 * (backward) j, then an IEEE division by the diagonal. */
void orc_spotrs_simt(int n, int nrhs, const float *a, int lda, float *b, int ldb, int upper)
{
    for (int r = 0; r < nrhs; ++r)
    {
        float *pb = b + (int64_t)r * ldb;
        for (int i = 0; i < n; ++i)
        {
            float x = pb[i];
            for (int j = 0; j < i; ++j) x = fmaf(-a[tri_at(lda, upper, i, j)], pb[j], x);
            pb[i] = x / a[(int64_t)i * (lda + 1)];
        }
        for (int i = n - 1; i >= 0; --i)
        {
            float x = pb[i];
            for (int j = i + 1; j < n; ++j) x = fmaf(-a[tri_at(lda, upper, j, i)], pb[j], x);
            pb[i] = x / a[(int64_t)i * (lda + 1)];
        }
    }
}

/* VectorTriSolve with AccumulateDot (cholesky_vector.cpp:30-122), used for 33..128 with one
 * right-hand side: a dot accumulator starts at zero and takes dot_i = fmaf(l, x_k, dot_i)
 * right-looking; each x_k = (b_k - dot_k) / l_kk, subtracted once. */
void orc_spotrs_dot(int n, int nrhs, const float *a, int lda, float *b, int ldb, int upper)
{
    float *dot = (float *)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    for (int r = 0; r < nrhs; ++r)
    {
        float *pb = b + (int64_t)r * ldb;
        for (int i = 0; i < n; ++i) dot[i] = 0.0f;
        for (int k = 0; k < n; ++k)
        {
            float x = (pb[k] - dot[k]) / a[(int64_t)k * (lda + 1)];
            pb[k] = x;
            for (int i = k + 1; i < n; ++i) dot[i] = fmaf(a[tri_at(lda, upper, i, k)], x, dot[i]);
        }
        for (int i = 0; i < n; ++i) dot[i] = 0.0f;
        for (int k = n - 1; k >= 0; --k)
        {
            float x = (pb[k] - dot[k]) / a[(int64_t)k * (lda + 1)];
            pb[k] = x;
            for (int i = 0; i < k; ++i) dot[i] = fmaf(a[tri_at(lda, upper, k, i)], x, dot[i]);
        }
    }
    free(dot);
}

/* n > 128 (this build's order; the reference solves panels with a Cube product here):
 * right-looking sweeps in blocks of ORC_NB rows.  Forward, per block [K0, K0 + w): the
 * block's unknowns x_k = x_k / l_kk in ascending k, each taken into the block's later rows
 * by fmaf(-l_ik, x_k, x_i); then every row below takes the block as one partial sum
 * t = fmaf(l_ik, x_k, t) from zero in ascending k, x_i = x_i - t.  Backward, blocks in
 * descending order: x_k = x_k / l_kk in descending k, taken into the block's earlier rows by
 * fmaf(-l_ki, x_k, x_i); every row above takes t = fmaf(l_ki, x_k, t) over the block in
 * ascending k, x_i = x_i - t. */
void orc_spotrs_right(int n, int nrhs, const float *a, int lda, float *b, int ldb, int upper)
{
    for (int r = 0; r < nrhs; ++r)
    {
        float *x = b + (int64_t)r * ldb;
        for (int K0 = 0; K0 < n; K0 += ORC_NB)
        {
            const int kend = K0 + ORC_NB < n ? K0 + ORC_NB : n;
            for (int k = K0; k < kend; ++k)
            {
                x[k] = x[k] / a[(int64_t)k * (lda + 1)];
                for (int i = k + 1; i < kend; ++i) x[i] = fmaf(-a[tri_at(lda, upper, i, k)], x[k], x[i]);
            }
            for (int i = kend; i < n; ++i)
            {
                float t = 0.0f;
                for (int k = K0; k < kend; ++k) t = fmaf(a[tri_at(lda, upper, i, k)], x[k], t);
                x[i] = x[i] - t;
            }
        }
        for (int K0 = ((n - 1) / ORC_NB) * ORC_NB; n > 0 && K0 >= 0; K0 -= ORC_NB)
        {
            const int kend = K0 + ORC_NB < n ? K0 + ORC_NB : n;
            for (int k = kend - 1; k >= K0; --k)
            {
                x[k] = x[k] / a[(int64_t)k * (lda + 1)];
                for (int i = K0; i < k; ++i) x[i] = fmaf(-a[tri_at(lda, upper, k, i)], x[k], x[i]);
            }
            for (int i = 0; i < K0; ++i)
            {
                float t = 0.0f;
                for (int k = K0; k < kend; ++k) t = fmaf(a[tri_at(lda, upper, k, i)], x[k], t);
                x[i] = x[i] - t;
            }
        }
    }
}

/* The solve dispatch of this build (cholesky_simt.cpp:186-199 with the batch always
 * larger than the reference's core count): batched n <= 32 and single n <= 8 use the
 * SolveKernel order; batched 33..128 and single 9..128 use the dot-accumulate order;
 * above 128 the right-looking order. */
void orc_spotrs(int n, int nrhs, const float *a, int lda, float *b, int ldb, int upper, int single)
{
    if (n > 128)
        orc_spotrs_right(n, nrhs, a, lda, b, ldb, upper);
    else if (single ? n > 8 : n > 32)
        orc_spotrs_dot(n, nrhs, a, lda, b, ldb, upper);
    else
        orc_spotrs_simt(n, nrhs, a, lda, b, ldb, upper);
}

/* ---------------------------------------------------------------------------------------
 * Real LU
 * ------------------------------------------------------------------------------------- */

/* Pivot row for column k (real_lu.hpp:59-139, PivotRF/PivotLocalRF): the first row with the
 * largest |a| among rows k..m-1; a NaN in row k keeps row k; other NaNs never win. */
static int lu_pivot(const float *col, int k, int m)
{
    float initial = col[k];
    if (initial != initial) return k;
    float best = fabsf(initial);
    int row = k;
    for (int i = k + 1; i < m; ++i)
    {
        float value = fabsf(col[i]);
        if (value > best)
        {
            best = value;
            row = i;
        }
    }
    return row;
}

/* P*A = L*U in place (FactorLocalCore, real_lu.hpp:409-448).  ipiv may be NULL (no
 * pivoting).  Returns info = first k+1 with U(k,k) == 0; such a column is neither scaled
 * nor used for updates. */
int orc_sgetrf(int m, int n, float *a, int lda, int *ipiv)
{
    int info = 0;
    int steps = m < n ? m : n;
    for (int k = 0; k < steps; ++k)
    {
        float *col = a + (int64_t)k * lda;
        int p = ipiv ? lu_pivot(col, k, m) : k;
        if (ipiv) ipiv[k] = p + 1;
        if (p != k)
            for (int j = 0; j < n; ++j)
            {
                float t = a[(int64_t)j * lda + k];
                a[(int64_t)j * lda + k] = a[(int64_t)j * lda + p];
                a[(int64_t)j * lda + p] = t;
            }
        float diagonal = col[k];
        if (diagonal == 0)
        {
            if (info == 0) info = k + 1;
            continue;
        }
        if (k + 1 == m) continue;
        for (int i = k + 1; i < m; ++i) col[i] = col[i] / diagonal;
        for (int j = k + 1; j < n; ++j)
        {
            float *cj = a + (int64_t)j * lda;
            float u = cj[k];
            for (int i = k + 1; i < m; ++i) cj[i] = fmaf(-col[i], u, cj[i]);
        }
    }
    return info;
}

/* Inverse from packed LU (real_lu_blocked_inverse_kernel.cpp): the permutation is the
 * identity with the pivot swaps applied in order (:676-714); info is the first zero U
 * diagonal, a failed matrix stores nothing (:716-738, :958-961); reciprocals r_k = 1/U(k,k)
 * by IEEE division; column c solves rhs = e with rhs[row] = (perm[row] == c); forward
 * rhs_i = fmaf(-rhs_k, L(i,k), rhs_i) for i > k, k ascending; backward s = rhs_k * r_k,
 * rhs_k = s, rhs_i = fmaf(-s, U(i,k), rhs_i) for i < k, k descending (:766-830). */
int orc_sgetri_vector(int n, const float *lu, int lda, const int *ipiv, float *c, int ldc)
{
    int info = 0;
    for (int k = 0; k < n; ++k)
        if (lu[(int64_t)k * (lda + 1)] == 0.0f)
        {
            info = k + 1;
            break;
        }
    if (info) return info;
    int *perm = (int *)malloc(sizeof(int) * (size_t)n);
    float *rec = (float *)malloc(sizeof(float) * (size_t)n);
    float *rhs = (float *)malloc(sizeof(float) * (size_t)n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    if (ipiv)
        for (int k = 0; k < n; ++k)
        {
            int p = ipiv[k] - 1;
            int t = perm[k];
            perm[k] = perm[p];
            perm[p] = t;
        }
    for (int k = 0; k < n; ++k) rec[k] = 1.0f / lu[(int64_t)k * (lda + 1)];
    for (int col = 0; col < n; ++col)
    {
        for (int i = 0; i < n; ++i) rhs[i] = perm[i] == col ? 1.0f : 0.0f;
        for (int k = 0; k < n; ++k)
        {
            float s = rhs[k];
            for (int i = k + 1; i < n; ++i) rhs[i] = fmaf(-s, lu[(int64_t)k * lda + i], rhs[i]);
        }
        for (int k = n - 1; k >= 0; --k)
        {
            float s = rhs[k] * rec[k];
            rhs[k] = s;
            for (int i = 0; i < k; ++i) rhs[i] = fmaf(-s, lu[(int64_t)k * lda + i], rhs[i]);
        }
        for (int i = 0; i < n; ++i) c[(int64_t)col * ldc + i] = rhs[i];
    }
    free(perm);
    free(rec);
    free(rhs);
    return 0;
}

/* LU solve, this build's order (the reference solve kernel is a CANN matmul chain; its
 * test reference is the numpy solve_lu of test/utils/lu_verify_utils.py:67-192, whose
 * mathematics this follows).  trans 0: row swaps k = 0..n-1, unit-lower forward
 * b_i = fmaf(-L(i,k), b_k, b_i) for i > k, k ascending; upper backward b_k = b_k / U(k,k),
 * b_i = fmaf(-U(i,k), b_k, b_i) for i < k, k descending.  trans 1: U^T w = b forward
 * (w_k = w_k / U(k,k), w_i = fmaf(-U(k,i), w_k, w_i), i > k), L^T z = w backward
 * (z_i = fmaf(-L(k,i), z_k, z_i), i < k, k descending), then the swaps in reverse order. */
void orc_sgetrs(int trans, int n, int nrhs, const float *lu, int lda, const int *ipiv, float *b, int ldb)
{
    for (int r = 0; r < nrhs; ++r)
    {
        float *x = b + (int64_t)r * ldb;
        if (trans == 0)
        {
            if (ipiv)
                for (int k = 0; k < n; ++k)
                {
                    int p = ipiv[k] - 1;
                    float t = x[k];
                    x[k] = x[p];
                    x[p] = t;
                }
            for (int k = 0; k < n; ++k)
                for (int i = k + 1; i < n; ++i) x[i] = fmaf(-lu[(int64_t)k * lda + i], x[k], x[i]);
            for (int k = n - 1; k >= 0; --k)
            {
                x[k] = x[k] / lu[(int64_t)k * (lda + 1)];
                for (int i = 0; i < k; ++i) x[i] = fmaf(-lu[(int64_t)k * lda + i], x[k], x[i]);
            }
        }
        else
        {
            for (int k = 0; k < n; ++k)
            {
                x[k] = x[k] / lu[(int64_t)k * (lda + 1)];
                for (int i = k + 1; i < n; ++i) x[i] = fmaf(-lu[(int64_t)i * lda + k], x[k], x[i]);
            }
            for (int k = n - 1; k >= 0; --k)
                for (int i = 0; i < k; ++i) x[i] = fmaf(-lu[(int64_t)i * lda + k], x[k], x[i]);
            if (ipiv)
                for (int k = n - 1; k >= 0; --k)
                {
                    int p = ipiv[k] - 1;
                    float t = x[k];
                    x[k] = x[p];
                    x[p] = t;
                }
        }
    }
}

/* ---------------------------------------------------------------------------------------
 * Complex64 Cholesky (this build's order; the reference keeps a compensated double-float
 * first column and diagonal, src/cpotrf/arch35/cholesky_factor.cpp:17-215, and uses a
 * CATLASS complex GEMM for n > 64, so the CUDA kernels and this restatement share the order
 * below and parity with the reference is by tolerance).  Interleaved (re, im) floats.
 * ------------------------------------------------------------------------------------- */

/* Element (i, j), j <= i, of the lower factor; upper storage holds the conjugate mirror. */
static inline void ctri_get(const float *a, int lda, int upper, int i, int j, float *re, float *im)
{
    if (upper)
    {
        const float *p = a + 2 * ((int64_t)i * lda + j);
        *re = p[0];
        *im = -p[1];
    }
    else
    {
        const float *p = a + 2 * ((int64_t)j * lda + i);
        *re = p[0];
        *im = p[1];
    }
}
static inline void ctri_set(float *a, int lda, int upper, int i, int j, float re, float im)
{
    if (upper)
    {
        float *p = a + 2 * ((int64_t)i * lda + j);
        p[0] = re;
        p[1] = -im;
    }
    else
    {
        float *p = a + 2 * ((int64_t)j * lda + i);
        p[0] = re;
        p[1] = im;
    }
}

/* Right-looking: d = Re(a_kk) (d > 0 and finite), s = sqrtf(d), l_kk = (s, 0),
 * l_ik = a_ik / s per component; a_ij -= l_ik conj(l_jk) as
 * re = fmaf(-ar, cr, re); re = fmaf(-ai, ci, re); im = fmaf(-ai, cr, im); im = fmaf(ar, ci, im). */
static int orc_cpotrf_seq(int n, float *a, int lda, int upper)
{
    float *w = (float *)malloc(sizeof(float) * 2 * (size_t)n * (size_t)n + 8);
    for (int j = 0; j < n; ++j)
        for (int i = j; i < n; ++i) ctri_get(a, lda, upper, i, j, &w[2 * ((size_t)j * n + i)], &w[2 * ((size_t)j * n + i) + 1]);
    int failure = 0;
    for (int k = 0; k < n; ++k)
    {
        float d = w[2 * ((size_t)k * n + k)];
        if (!(d > 0.0f && d <= FLT_MAX_VALUE))
        {
            failure = k + 1;
            break;
        }
        float s = sqrtf(d);
        w[2 * ((size_t)k * n + k)] = s;
        w[2 * ((size_t)k * n + k) + 1] = 0.0f;
        for (int i = k + 1; i < n; ++i)
        {
            float *v = &w[2 * ((size_t)k * n + i)];
            v[0] = v[0] / s;
            v[1] = v[1] / s;
        }
        for (int j = k + 1; j < n; ++j)
        {
            float cr = w[2 * ((size_t)k * n + j)], ci = w[2 * ((size_t)k * n + j) + 1];
            for (int i = j; i < n; ++i)
            {
                float ar = w[2 * ((size_t)k * n + i)], ai = w[2 * ((size_t)k * n + i) + 1];
                float *z = &w[2 * ((size_t)j * n + i)];
                float re = z[0], im = z[1];
                re = fmaf(-ar, cr, re);
                re = fmaf(-ai, ci, re);
                im = fmaf(-ai, cr, im);
                im = fmaf(ar, ci, im);
                z[0] = re;
                z[1] = im;
            }
        }
    }
    int done = failure ? failure - 1 : n;
    for (int j = 0; j < done; ++j)
        for (int i = j; i < n; ++i) ctri_set(a, lda, upper, i, j, w[2 * ((size_t)j * n + i)], w[2 * ((size_t)j * n + i) + 1]);
    free(w);
    return failure;
}

/* Right-looking sweeps: y_k = z_k / l_kk, z_i -= l_ik y_k (i > k); then x_k = z_k / l_kk,
 * z_i -= conj(l_ki) x_k (i < k, k descending); z -= l y as re = fmaf(-lr, yr, re);
 * re = fmaf(li, yi, re); im = fmaf(-lr, yi, im); im = fmaf(-li, yr, im). */
static void orc_cpotrs_seq(int n, int nrhs, const float *a, int lda, float *b, int ldb, int upper)
{
    for (int r = 0; r < nrhs; ++r)
    {
        float *x = b + 2 * (int64_t)r * ldb;
        for (int k = 0; k < n; ++k)
        {
            float dr, di;
            ctri_get(a, lda, upper, k, k, &dr, &di);
            float yr = x[2 * k] / dr, yi = x[2 * k + 1] / dr;
            for (int i = k + 1; i < n; ++i)
            {
                float lr, li;
                ctri_get(a, lda, upper, i, k, &lr, &li);
                float re = x[2 * i], im = x[2 * i + 1];
                re = fmaf(-lr, yr, re);
                re = fmaf(li, yi, re);
                im = fmaf(-lr, yi, im);
                im = fmaf(-li, yr, im);
                x[2 * i] = re;
                x[2 * i + 1] = im;
            }
            x[2 * k] = yr;
            x[2 * k + 1] = yi;
        }
        for (int k = n - 1; k >= 0; --k)
        {
            float dr, di;
            ctri_get(a, lda, upper, k, k, &dr, &di);
            float yr = x[2 * k] / dr, yi = x[2 * k + 1] / dr;
            for (int i = 0; i < k; ++i)
            {
                float lr, li;
                ctri_get(a, lda, upper, k, i, &lr, &li);
                li = -li; /* conj(l_ki) */
                float re = x[2 * i], im = x[2 * i + 1];
                re = fmaf(-lr, yr, re);
                re = fmaf(li, yi, re);
                im = fmaf(-lr, yi, im);
                im = fmaf(-li, yr, im);
                x[2 * i] = re;
                x[2 * i + 1] = im;
            }
            x[2 * k] = yr;
            x[2 * k + 1] = yi;
        }
    }
}

/* Above order 240 (the whole-GPU complex factorisation and the solve that goes with it):
 * the same arithmetic in 64-column panels with panel partial sums, as orc_spotrf_blocked.
 * Inside a panel: l_ik = a_ik / s, a_ij -= l_ik conj(l_jk) as the four FMAs above in
 * ascending k.  Right of the panel: t = sum_k l_ik conj(l_jk) from zero in ascending k,
 *   tr = fmaf(ar, cr, tr); tr = fmaf(ai, ci, tr); ti = fmaf(ai, cr, ti); ti = fmaf(-ar, ci, ti)
 * then a_ij = (re - tr, im - ti). */
static int orc_cpotrf_blocked(int n, float *a, int lda, int upper)
{
    float *w = (float *)malloc(sizeof(float) * 2 * (size_t)n * (size_t)n + 8);
#define W(i, j) (w + 2 * ((size_t)(j) * n + (i)))
    for (int j = 0; j < n; ++j)
        for (int i = j; i < n; ++i) ctri_get(a, lda, upper, i, j, W(i, j), W(i, j) + 1);
    int failure = 0;
    for (int k0 = 0; k0 < n && !failure; k0 += ORC_NB)
    {
        const int kend = k0 + ORC_NB < n ? k0 + ORC_NB : n;
        for (int k = k0; k < kend; ++k)
        {
            float d = W(k, k)[0];
            if (!(d > 0.0f && d <= FLT_MAX_VALUE))
            {
                failure = k + 1;
                break;
            }
            float s = sqrtf(d);
            W(k, k)[0] = s;
            W(k, k)[1] = 0.0f;
            for (int i = k + 1; i < n; ++i)
            {
                W(i, k)[0] = W(i, k)[0] / s;
                W(i, k)[1] = W(i, k)[1] / s;
            }
            for (int j = k + 1; j < kend; ++j)
            {
                const float cr = W(j, k)[0], ci = W(j, k)[1];
                for (int i = j; i < n; ++i)
                {
                    const float ar = W(i, k)[0], ai = W(i, k)[1];
                    float re = W(i, j)[0], im = W(i, j)[1];
                    re = fmaf(-ar, cr, re);
                    re = fmaf(-ai, ci, re);
                    im = fmaf(-ai, cr, im);
                    im = fmaf(ar, ci, im);
                    W(i, j)[0] = re;
                    W(i, j)[1] = im;
                }
            }
        }
        if (failure) break;
        for (int j = kend; j < n; ++j)
            for (int i = j; i < n; ++i)
            {
                float tr = 0.0f, ti = 0.0f;
                for (int k = k0; k < kend; ++k)
                {
                    const float ar = W(i, k)[0], ai = W(i, k)[1], cr = W(j, k)[0], ci = W(j, k)[1];
                    tr = fmaf(ar, cr, tr);
                    tr = fmaf(ai, ci, tr);
                    ti = fmaf(ai, cr, ti);
                    ti = fmaf(-ar, ci, ti);
                }
                W(i, j)[0] = W(i, j)[0] - tr;
                W(i, j)[1] = W(i, j)[1] - ti;
            }
    }
    int done = failure ? failure - 1 : n;
    for (int j = 0; j < done; ++j)
        for (int i = j; i < n; ++i) ctri_set(a, lda, upper, i, j, W(i, j)[0], W(i, j)[1]);
#undef W
    free(w);
    return failure;
}

/* The blocked solve above order 240, as orc_spotrs_right with complex products: inside a
 * block z_i -= l_ik y_k (the four FMAs of orc_cpotrs_seq), below it one partial sum
 *   tr = fmaf(lr, yr, tr); tr = fmaf(-li, yi, tr); ti = fmaf(lr, yi, ti); ti = fmaf(li, yr, ti)
 * from zero in ascending k, then z_i = (re - tr, im - ti); backward the same with conj(l_ki). */
static void orc_cpotrs_blocked(int n, int nrhs, const float *a, int lda, float *b, int ldb, int upper)
{
    for (int r = 0; r < nrhs; ++r)
    {
        float *x = b + 2 * (int64_t)r * ldb;
        for (int K0 = 0; K0 < n; K0 += ORC_NB)
        {
            const int kend = K0 + ORC_NB < n ? K0 + ORC_NB : n;
            for (int k = K0; k < kend; ++k)
            {
                float dr, di;
                ctri_get(a, lda, upper, k, k, &dr, &di);
                const float yr = x[2 * k] / dr, yi = x[2 * k + 1] / dr;
                for (int i = k + 1; i < kend; ++i)
                {
                    float lr, li;
                    ctri_get(a, lda, upper, i, k, &lr, &li);
                    float re = x[2 * i], im = x[2 * i + 1];
                    re = fmaf(-lr, yr, re);
                    re = fmaf(li, yi, re);
                    im = fmaf(-lr, yi, im);
                    im = fmaf(-li, yr, im);
                    x[2 * i] = re;
                    x[2 * i + 1] = im;
                }
                x[2 * k] = yr;
                x[2 * k + 1] = yi;
            }
            for (int i = kend; i < n; ++i)
            {
                float tr = 0.0f, ti = 0.0f;
                for (int k = K0; k < kend; ++k)
                {
                    float lr, li;
                    ctri_get(a, lda, upper, i, k, &lr, &li);
                    const float yr = x[2 * k], yi = x[2 * k + 1];
                    tr = fmaf(lr, yr, tr);
                    tr = fmaf(-li, yi, tr);
                    ti = fmaf(lr, yi, ti);
                    ti = fmaf(li, yr, ti);
                }
                x[2 * i] = x[2 * i] - tr;
                x[2 * i + 1] = x[2 * i + 1] - ti;
            }
        }
        for (int K0 = ((n - 1) / ORC_NB) * ORC_NB; n > 0 && K0 >= 0; K0 -= ORC_NB)
        {
            const int kend = K0 + ORC_NB < n ? K0 + ORC_NB : n;
            for (int k = kend - 1; k >= K0; --k)
            {
                float dr, di;
                ctri_get(a, lda, upper, k, k, &dr, &di);
                const float yr = x[2 * k] / dr, yi = x[2 * k + 1] / dr;
                for (int i = K0; i < k; ++i)
                {
                    float lr, li;
                    ctri_get(a, lda, upper, k, i, &lr, &li);
                    li = -li; /* conj(l_ki) */
                    float re = x[2 * i], im = x[2 * i + 1];
                    re = fmaf(-lr, yr, re);
                    re = fmaf(li, yi, re);
                    im = fmaf(-lr, yi, im);
                    im = fmaf(-li, yr, im);
                    x[2 * i] = re;
                    x[2 * i + 1] = im;
                }
                x[2 * k] = yr;
                x[2 * k + 1] = yi;
            }
            for (int i = 0; i < K0; ++i)
            {
                float tr = 0.0f, ti = 0.0f;
                for (int k = K0; k < kend; ++k)
                {
                    float lr, li;
                    ctri_get(a, lda, upper, k, i, &lr, &li);
                    li = -li; /* conj(l_ki) */
                    const float yr = x[2 * k], yi = x[2 * k + 1];
                    tr = fmaf(lr, yr, tr);
                    tr = fmaf(-li, yi, tr);
                    ti = fmaf(lr, yi, ti);
                    ti = fmaf(li, yr, ti);
                }
                x[2 * i] = x[2 * i] - tr;
                x[2 * i + 1] = x[2 * i + 1] - ti;
            }
        }
    }
}

/* The complex dispatch of this build: the block and register paths up to order 240, the
 * whole-GPU blocked order above. */
int orc_cpotrf(int n, float *a, int lda, int upper)
{
    return n > 240 ? orc_cpotrf_blocked(n, a, lda, upper) : orc_cpotrf_seq(n, a, lda, upper);
}
void orc_cpotrs(int n, int nrhs, const float *a, int lda, float *b, int ldb, int upper)
{
    if (n > 240)
        orc_cpotrs_blocked(n, nrhs, a, lda, b, ldb, upper);
    else
        orc_cpotrs_seq(n, nrhs, a, lda, b, ldb, upper);
}

/* ---------------------------------------------------------------------------------------
 * Batched drivers over a contiguous slab (matrix b at base + b*stride), OpenMP over
 * matrices; `threads` <= 0 uses the OpenMP default.  These are what the CPU baseline times.
 * ------------------------------------------------------------------------------------- */

static void set_threads(int threads)
{
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
}

int orc_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_spotrf_batched(int n, float *a, int lda, int64_t stride, int count, int upper, int *info, int threads)
{
    set_threads(threads);
#pragma omp parallel for schedule(static)
    for (int q = 0; q < count; ++q) info[q] = orc_spotrf(n, a + (int64_t)q * stride, lda, upper);
}

void orc_spotrs_batched(int n, int nrhs, const float *a, int lda, int64_t astride, float *b, int ldb,
                        int64_t bstride, int count, int upper, int single, int threads)
{
    set_threads(threads);
#pragma omp parallel for schedule(static)
    for (int q = 0; q < count; ++q)
        orc_spotrs(n, nrhs, a + (int64_t)q * astride, lda, b + (int64_t)q * bstride, ldb, upper, single);
}

void orc_sgetrf_batched(int m, int n, float *a, int lda, int64_t stride, int count, int *ipiv, int *info,
                        int threads)
{
    set_threads(threads);
    int steps = m < n ? m : n;
#pragma omp parallel for schedule(static)
    for (int q = 0; q < count; ++q)
        info[q] = orc_sgetrf(m, n, a + (int64_t)q * stride, lda, ipiv ? ipiv + (int64_t)q * steps : NULL);
}

void orc_sgetrs_batched(int trans, int n, int nrhs, const float *lu, int lda, int64_t astride, const int *ipiv,
                        float *b, int ldb, int64_t bstride, int count, int threads)
{
    set_threads(threads);
#pragma omp parallel for schedule(static)
    for (int q = 0; q < count; ++q)
        orc_sgetrs(trans, n, nrhs, lu + (int64_t)q * astride, lda, ipiv ? ipiv + (int64_t)q * n : NULL,
                   b + (int64_t)q * bstride, ldb);
}

void orc_sgetri_batched(int n, const float *lu, int lda, int64_t astride, const int *ipiv, float *c, int ldc,
                        int64_t cstride, int count, int *info, int threads)
{
    set_threads(threads);
#pragma omp parallel for schedule(static)
    for (int q = 0; q < count; ++q)
        info[q] = orc_sgetri_vector(n, lu + (int64_t)q * astride, lda, ipiv ? ipiv + (int64_t)q * n : NULL,
                                    c + (int64_t)q * cstride, ldc);
}

/* Complex batches: matrix q at a + 2*q*astride floats (astride in complex elements). */
void orc_cpotrf_batched(int n, float *a, int lda, int64_t stride, int count, int upper, int *info, int threads)
{
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 16)
    for (int q = 0; q < count; ++q) info[q] = orc_cpotrf(n, a + 2 * (int64_t)q * stride, lda, upper);
}

void orc_cpotrs_batched(int n, int nrhs, const float *a, int lda, int64_t astride, float *b, int ldb,
                        int64_t bstride, int count, int upper, int threads)
{
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 16)
    for (int q = 0; q < count; ++q)
        orc_cpotrs(n, nrhs, a + 2 * (int64_t)q * astride, lda, b + 2 * (int64_t)q * bstride, ldb, upper);
}

/* ---------------------------------------------------------------------------------------
 * Complex LU family (complex64 stored as interleaved float pairs, column-major)
 *
 * Restated from the reference's SIMT helpers (paths relative to the reference root):
 *   c_score            src/utils/complex_solver_kernel.hpp:48-67   (PivotScore)
 *   c_submul           :69-72                                     (SubMul)
 *   c_quotient         :74-86                                     (Quotient)
 *   c_scaled_quotient  :88-106                                    (ScaledQuotient)
 *   c_needs_scaled     :108-117                                   (NeedsScaledNumerator)
 *   c_divide           :119-143                                   (Divide)
 *   orc_cgetrf         :161-250 (FindPivot, SwapRows, DivideColumn, UpdatePanel,
 *                      FactorColumn): every element receives its SubMul updates one
 *                      pivot at a time in ascending order, so the reference's panel,
 *                      cached-panel and vector trailing-update schedules all give these bits
 *   orc_cgetri         src/utils/complex_solver_resident.hpp:21-170 (CompensatedSubtract,
 *                      CompensatedSubMul, WarpResidentStep / WarpResidentSolve) with
 *                      ParallelCheckLu (complex_solver_kernel.hpp:262-292)
 *   orc_cmatinv        src/utils/complex_solver_register.hpp:271-326 (InvertSmallInPlace,
 *                      SolveDirectInPlace: Gauss-Jordan in place, then the column permutation)
 *   orc_cgetrs         this build's own order (the reference hands its solve to Cube
 *                      matrix multiplies, src/cgetrs/kernel/trsm_custom.hpp): pivots, then
 *                      per-element SubMul chains in pivot order, Divide by the diagonal
 * ------------------------------------------------------------------------------------- */

typedef struct
{
    float re, im;
} cfl;

static inline uint32_t c_bits(float x)
{
    uint32_t u;
    memcpy(&u, &x, sizeof u);
    return u;
}

static inline float c_float(uint32_t u)
{
    float x;
    memcpy(&x, &u, sizeof x);
    return x;
}

/* Abs keeps the sign of a negative zero (x < 0 is false for -0). */
static inline float c_abs(float x) { return x < 0.0f ? -x : x; }

static inline int c_zero(cfl v) { return v.re == 0.0f && v.im == 0.0f; }

/* L1 magnitude as an ordered key: NaN 0, zero 1, an overflowing sum re-scaled by 1/2 with
 * its exponent extended by one. */
static inline uint32_t c_score(cfl v)
{
    float re = c_abs(v.re), im = c_abs(v.im);
    float s = re + im;
    if (!(s >= 0.0f)) return 0u;
    if (s == 0.0f) return 1u;
    if (s > FLT_MAX_VALUE) return c_bits(re * 0.5f + im * 0.5f) + 0x00800001u;
    return c_bits(s) + 1u;
}

/* x - a*b with the reference's two-FMA order per component. */
static inline cfl c_submul(cfl x, cfl a, cfl b)
{
    cfl r;
    r.re = fmaf(a.im, b.im, fmaf(-a.re, b.re, x.re));
    r.im = fmaf(-a.im, b.re, fmaf(-a.re, b.im, x.im));
    return r;
}

static inline float c_quotient(float ar, float br, float ai, float bi, float den, float den_err)
{
    float product = ar * br;
    float other = ai * bi;
    float numerator = product + other;
    float part = numerator - product;
    float error = (product - (numerator - part)) + (other - part) + fmaf(ar, br, -product) + fmaf(ai, bi, -other);
    float reciprocal = 1.0f / den;
    float result = numerator * reciprocal;
    float remainder = fmaf(-result, den, numerator) + error - result * den_err;
    return fmaf(remainder, reciprocal, result);
}

static inline float c_scaled_quotient(float a, float b, float c, float d, float scale, float den, float den_err)
{
    int ae, be, ce, de, se;
    float am = frexpf(a, &ae), bm = frexpf(b, &be);
    float cm = frexpf(c, &ce), dm = frexpf(d, &de);
    float sm = frexpf(scale, &se);
    int ab = ae + be, cd = ce + de;
    int zab = a == 0.0f || b == 0.0f, zcd = c == 0.0f || d == 0.0f;
    int e = zab ? cd : zcd ? ab : (ab > cd ? ab : cd);
    am = zab ? 0.0f : ldexpf(am, ab - e);
    cm = zcd ? 0.0f : ldexpf(cm, cd - e);
    float q = c_quotient(am, bm, cm, dm, den, den_err);
    return ldexpf(q / (sm * sm), e - 2 * se);
}

static inline int c_needs_scaled(cfl a, cfl b, float scale, float ar, float ai)
{
    return c_abs(a.re) <= FLT_MAX_VALUE && c_abs(a.im) <= FLT_MAX_VALUE && scale > 0.0f && scale <= FLT_MAX_VALUE &&
           (c_abs(ar) > 0x1p120f || c_abs(ai) > 0x1p120f || (a.re != 0.0f && c_abs(ar) < 0x1p-100f) ||
            (a.im != 0.0f && c_abs(ai) < 0x1p-100f) || (b.re != 0.0f && c_abs(b.re / scale) < 0x1p-100f) ||
            (b.im != 0.0f && c_abs(b.im / scale) < 0x1p-100f));
}

/* a / b: both scaled by the exponent of max(|b.re|, |b.im|), the compensated quotient, and
 * exponent-aligned products when the scaled operands would lose bits. */
static cfl c_divide(cfl a, cfl b)
{
    float s = c_abs(b.re) > c_abs(b.im) ? c_abs(b.re) : c_abs(b.im);
    uint32_t ex = c_bits(s) & 0x7f800000u;
    if (ex != 0) s = c_float(ex);
    float br = b.re / s, bi = b.im / s, ar = a.re / s, ai = a.im / s;
    float first = c_abs(br) > c_abs(bi) ? br : bi;
    float second = c_abs(br) > c_abs(bi) ? bi : br;
    float square = first * first;
    float den = fmaf(second, second, square);
    float err = fmaf(first, first, -square) + fmaf(second, second, square - den);
    cfl r;
    if (c_needs_scaled(a, b, s, ar, ai))
    {
        r.re = c_scaled_quotient(a.re, b.re, a.im, b.im, s, den, err);
        r.im = c_scaled_quotient(a.im, b.re, -a.re, b.im, s, den, err);
        return r;
    }
    r.re = c_quotient(ar, br, ai, bi, den, err);
    r.im = c_quotient(ai, br, -ar, bi, den, err);
    return r;
}

#define CAT(a, lda, r, c) ((a)[(int64_t)(c) * (lda) + (r)])

/* In-place LU of the m x n matrix; ipiv NULL selects no pivoting.  Returns info: the first
 * column whose pivot is exactly zero, 1-based, or 0. */
int orc_cgetrf(int m, int n, float *af, int lda, int *ipiv)
{
    cfl *a = (cfl *)af;
    int info = 0, lim = m < n ? m : n;
    for (int k = 0; k < lim; ++k)
    {
        int p = k;
        if (ipiv)
        {
            uint32_t best = 0;
            p = m;
            for (int r = k; r < m; ++r)
            {
                uint32_t s = c_score(CAT(a, lda, r, k));
                if (s > best || (s == best && r < p))
                {
                    best = s;
                    p = r;
                }
            }
            ipiv[k] = p + 1;
        }
        if (info == 0 && c_zero(CAT(a, lda, p, k))) info = k + 1;
        if (p != k)
            for (int j = 0; j < n; ++j)
            {
                cfl t = CAT(a, lda, k, j);
                CAT(a, lda, k, j) = CAT(a, lda, p, j);
                CAT(a, lda, p, j) = t;
            }
        cfl d = CAT(a, lda, k, k);
        if (!c_zero(d))
            for (int r = k + 1; r < m; ++r) CAT(a, lda, r, k) = c_divide(CAT(a, lda, r, k), d);
        for (int j = k + 1; j < n; ++j)
        {
            cfl u = CAT(a, lda, k, j);
            for (int r = k + 1; r < m; ++r) CAT(a, lda, r, j) = c_submul(CAT(a, lda, r, j), CAT(a, lda, r, k), u);
        }
    }
    return info;
}

/* Status of an LU ahead of its inverse: -4 for a pivot outside [row+1, n], else the first
 * exactly-zero diagonal (1-based), else 0. */
int orc_ccheck_lu(int n, const float *lu, int lda, const int *ipiv)
{
    const cfl *a = (const cfl *)lu;
    if (ipiv)
        for (int r = 0; r < n; ++r)
            if (ipiv[r] < r + 1 || ipiv[r] > n) return -4;
    for (int r = 0; r < n; ++r)
        if (c_zero(CAT(a, lda, r, r))) return r + 1;
    return 0;
}

/* value - left*right, its rounding error carried into *corr. */
static inline float c_comp_sub(float value, float *corr, float left, float right)
{
    float product = left * right;
    float product_err = fmaf(left, right, -product);
    float result = value - product;
    float virt = result - value;
    float sum_err = (value - (result - virt)) - (product + virt);
    *corr += sum_err - product_err;
    return result;
}

static inline void c_comp_submul(cfl *v, cfl *corr, cfl f, cfl s)
{
    v->re = c_comp_sub(v->re, &corr->re, f.re, s.re);
    v->re = c_comp_sub(v->re, &corr->re, -f.im, s.im);
    v->im = c_comp_sub(v->im, &corr->im, f.im, s.re);
    v->im = c_comp_sub(v->im, &corr->im, f.re, s.im);
}

/* Inverse from an LU: column j solves L U x = P e_j with compensated updates.  C is written
 * only when the LU check passes.  Returns the check status. */
int orc_cgetri(int n, const float *lu, int lda, const int *ipiv, float *cf_, int ldc)
{
    const cfl *a = (const cfl *)lu;
    cfl *c = (cfl *)cf_;
    int status = orc_ccheck_lu(n, lu, lda, ipiv);
    if (status != 0) return status;
    int *perm = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    cfl *x = (cfl *)malloc(sizeof(cfl) * 2 * (size_t)(n > 0 ? n : 1));
    cfl *e = x + n;
    for (int r = 0; r < n; ++r) perm[r] = r;
    if (ipiv)
        for (int r = 0; r < n; ++r)
        {
            int t = ipiv[r] - 1, v = perm[r];
            perm[r] = perm[t];
            perm[t] = v;
        }
    for (int j = 0; j < n; ++j)
    {
        for (int r = 0; r < n; ++r)
        {
            x[r].re = perm[r] == j ? 1.0f : 0.0f;
            x[r].im = 0.0f;
            e[r].re = e[r].im = 0.0f;
        }
        for (int p = 0; p < n; ++p)
        {
            cfl v = {x[p].re + e[p].re, x[p].im + e[p].im};
            for (int r = p + 1; r < n; ++r) c_comp_submul(&x[r], &e[r], CAT(a, lda, r, p), v);
        }
        for (int p = n - 1; p >= 0; --p)
        {
            cfl v = {x[p].re + e[p].re, x[p].im + e[p].im};
            v = c_divide(v, CAT(a, lda, p, p));
            x[p] = v;
            e[p].re = e[p].im = 0.0f;
            for (int r = 0; r < p; ++r) c_comp_submul(&x[r], &e[r], CAT(a, lda, r, p), v);
        }
        for (int r = 0; r < n; ++r) CAT(c, ldc, r, j) = x[r];
    }
    free(x);
    free(perm);
    return 0;
}

/* Gauss-Jordan inverse in place with partial pivoting (n <= 32 in the API).  An exactly
 * zero pivot stops the sweep and returns its column, 1-based, with C unwritten. */
int orc_cmatinv(int n, const float *af, int lda, float *cf_, int ldc)
{
    const cfl *a = (const cfl *)af;
    cfl *c = (cfl *)cf_;
    size_t nn = (size_t)(n > 0 ? n : 1);
    cfl *w = (cfl *)malloc(sizeof(cfl) * nn * nn);
    cfl *upper = (cfl *)malloc(sizeof(cfl) * nn);
    int *piv = (int *)malloc(sizeof(int) * nn);
    int status = 0;
    for (int j = 0; j < n; ++j)
        for (int r = 0; r < n; ++r) CAT(w, n, r, j) = CAT(a, lda, r, j);
    for (int col = 0; col < n && status == 0; ++col)
    {
        uint32_t best = 0;
        int p = col;
        for (int r = col; r < n; ++r)
        {
            uint32_t s = c_score(CAT(w, n, r, col));
            if (s > best)
            {
                best = s;
                p = r;
            }
        }
        piv[col] = p;
        for (int j = 0; j < n; ++j)
        {
            cfl t = CAT(w, n, col, j);
            CAT(w, n, col, j) = CAT(w, n, p, j);
            CAT(w, n, p, j) = t;
        }
        cfl d = CAT(w, n, col, col);
        if (c_zero(d))
        {
            status = col + 1;
            break;
        }
        cfl one = {1.0f, 0.0f};
        cfl inv = c_divide(one, d);
        for (int j = 0; j < n; ++j) upper[j] = j == col ? inv : c_divide(CAT(w, n, col, j), d);
        for (int j = 0; j < n; ++j) CAT(w, n, col, j) = upper[j];
        for (int r = 0; r < n; ++r)
        {
            if (r == col) continue;
            cfl f = CAT(w, n, r, col);
            for (int j = 0; j < n; ++j)
            {
                if (j == col)
                {
                    cfl v;
                    v.re = fmaf(f.im, inv.im, -f.re * inv.re);
                    v.im = fmaf(-f.re, inv.im, -f.im * inv.re);
                    CAT(w, n, r, j) = v;
                }
                else
                    CAT(w, n, r, j) = c_submul(CAT(w, n, r, j), f, upper[j]);
            }
        }
    }
    if (status == 0)
        for (int col = 0; col < n; ++col)
        {
            int t = col;
            for (int r = n - 1; r >= 0; --r)
            {
                int q = piv[r];
                t = t == r ? q : t == q ? r : t;
            }
            for (int r = 0; r < n; ++r) CAT(c, ldc, r, t) = CAT(w, n, r, col);
        }
    free(piv);
    free(upper);
    free(w);
    return status;
}

/* Solve with an LU: trans 0 A X = B, 1 A^T X = B, 2 A^H X = B.  The working triangle is
 * M = A (trans 0) or op(A) (trans 1, 2); every element of B receives its SubMul updates in
 * pivot order and is divided by the diagonal of the non-unit factor after them. */
void orc_cgetrs(int trans, int n, int nrhs, const float *lu, int lda, const int *ipiv, float *bf, int ldb)
{
    const cfl *a = (const cfl *)lu;
    cfl *b = (cfl *)bf;
    const float cj = trans == 2 ? -1.0f : 1.0f;
#define CM(r, c)                                                                                     \
    (trans == 0 ? CAT(a, lda, r, c)                                                                  \
                : (cfl){CAT(a, lda, c, r).re, cj * CAT(a, lda, c, r).im})
    for (int j = 0; j < nrhs; ++j)
    {
        cfl *x = b + (int64_t)j * ldb;
        if (trans == 0)
        {
            if (ipiv)
                for (int k = 0; k < n; ++k)
                {
                    int t = ipiv[k] - 1;
                    cfl v = x[k];
                    x[k] = x[t];
                    x[t] = v;
                }
            for (int k = 0; k < n; ++k)
                for (int i = k + 1; i < n; ++i) x[i] = c_submul(x[i], CM(i, k), x[k]);
            for (int k = n - 1; k >= 0; --k)
            {
                x[k] = c_divide(x[k], CM(k, k));
                for (int i = 0; i < k; ++i) x[i] = c_submul(x[i], CM(i, k), x[k]);
            }
        }
        else
        {
            for (int k = 0; k < n; ++k)
            {
                x[k] = c_divide(x[k], CM(k, k));
                for (int i = k + 1; i < n; ++i) x[i] = c_submul(x[i], CM(i, k), x[k]);
            }
            for (int k = n - 1; k >= 0; --k)
                for (int i = 0; i < k; ++i) x[i] = c_submul(x[i], CM(i, k), x[k]);
            if (ipiv)
                for (int k = n - 1; k >= 0; --k)
                {
                    int t = ipiv[k] - 1;
                    cfl v = x[k];
                    x[k] = x[t];
                    x[t] = v;
                }
        }
    }
#undef CM
}

/* Complex divide and pivot score exposed for the element-level parity tests. */
void orc_cdivide_many(const float *a, const float *b, float *out, int64_t count)
{
    for (int64_t i = 0; i < count; ++i)
    {
        cfl x = {a[2 * i], a[2 * i + 1]}, y = {b[2 * i], b[2 * i + 1]};
        cfl r = c_divide(x, y);
        out[2 * i] = r.re;
        out[2 * i + 1] = r.im;
    }
}

void orc_cgetrf_batched(int m, int n, float *a, int lda, int64_t stride, int count, int pivoting, int *ipiv,
                        int *info, int threads)
{
    int lim = m < n ? m : n;
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 4)
    for (int q = 0; q < count; ++q)
        info[q] = orc_cgetrf(m, n, a + 2 * (int64_t)q * stride, lda, pivoting ? ipiv + (int64_t)q * lim : NULL);
}

void orc_cgetri_batched(int n, const float *lu, int lda, int64_t astride, const int *ipiv, float *c, int ldc,
                        int64_t cstride, int count, int *info, int threads)
{
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 4)
    for (int q = 0; q < count; ++q)
        info[q] = orc_cgetri(n, lu + 2 * (int64_t)q * astride, lda, ipiv ? ipiv + (int64_t)q * n : NULL,
                             c + 2 * (int64_t)q * cstride, ldc);
}

void orc_cmatinv_batched(int n, const float *a, int lda, int64_t astride, float *c, int ldc, int64_t cstride,
                         int count, int *info, int threads)
{
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 64)
    for (int q = 0; q < count; ++q)
        info[q] = orc_cmatinv(n, a + 2 * (int64_t)q * astride, lda, c + 2 * (int64_t)q * cstride, ldc);
}

void orc_cgetrs_batched(int trans, int n, int nrhs, const float *lu, int lda, int64_t astride, const int *ipiv,
                        float *b, int ldb, int64_t bstride, int count, int threads)
{
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 4)
    for (int q = 0; q < count; ++q)
        orc_cgetrs(trans, n, nrhs, lu + 2 * (int64_t)q * astride, lda, ipiv ? ipiv + (int64_t)q * n : NULL,
                   b + 2 * (int64_t)q * bstride, ldb);
}

/* ---------------------------------------------------------------------------------------
 * Real QR family (Householder, column-major)
 *
 * The reference's CPU golden for its QR tests is QrCore::Larfg / Geqr2 / Larft
 * (src/sgeqrf/kernel/householder.hpp:55-200): LAPACK's sign convention (beta = -sign(alpha)
 * ||x||, tau = (beta - alpha) / beta, v = x2 / (alpha - beta), tau = 0 when x2 is zero).
 * Its device kernels hand the trailing products to the Cube unit, whose summation order is
 * not in its sources, so these routines state this build's blocked order, which the CUDA
 * kernels follow bit for bit:
 *   - every reduction over rows is a "lane sum": row r feeds partial r mod 32 (an FMA
 *     chain in ascending row order per partial), then the 32 partials are combined by a
 *     butterfly, p[l] = p[l] + p[l ^ off] for off = 16, 8, 4, 2, 1;
 *   - panels of 32 columns: Larfg per column, the reflector applied to the rest of the
 *     panel (w = tau * (v . a), a -= w v by FMA), the block factor T of slarft (forward,
 *     columnwise), then the trailing columns C -= V (T^T (V^T C)) with each W2 entry an FMA
 *     chain over T in ascending order and each C entry an FMA chain over the reflectors in
 *     ascending order;
 *   - orc_sgels: geqrf, Q^T B by the same block application, then R X = (Q^T B)(1:n) by a
 *     backward sweep (IEEE division, FMA updates in descending pivot order).
 * Outside the magnitude window 5e-20 < max|A| < 1.8e19 the squares overflow or underflow, as
 * in the reference kernels (no rescaling pass).
 * ------------------------------------------------------------------------------------- */

#define QR_NB 32
#define RAT(a, lda, r, c) ((a)[(int64_t)(c) * (lda) + (r)])

static float qr_lane_fold(float *p)
{
    for (int off = 16; off > 0; off >>= 1)
    {
        float q[32];
        for (int l = 0; l < 32; ++l) q[l] = p[l] + p[l ^ off];
        memcpy(p, q, sizeof q);
    }
    return p[0];
}

/* Reflector i of a panel starting at column k: v(row) = 1 at row k+i, A(row, k+i) below. */
static inline float qr_v(const float *a, int lda, int k, int i, int row)
{
    return row == k + i ? 1.0f : RAT(a, lda, row, k + i);
}

/* Rows per segment of a panel's reductions.  A panel (rows [k, m) of kb columns) that fits
 * one block's shared memory (budget elements) is reduced as one segment (0).  A larger one is
 * spread over an eight-block cluster: block s holds rows [k + s seg, k + (s + 1) seg), seg =
 * ceil((m - k) / 8) rounded up to a multiple of 32, and each reduction over rows becomes one
 * lane sum per segment, folded, with the segment totals added in ascending order.  A panel
 * too tall even for that is again one segment. */
static int qr_panel_seg(int H, int kb, int budget)
{
    if ((int64_t)H * kb <= budget) return 0;
    const int seg = ((H + 7) / 8 + 31) & ~31;
    return (int64_t)seg * kb <= budget ? seg : 0;
}

/* Folds the lane partials p of one segment into *total (segment totals in ascending order). */
static void qr_seg_flush(float *p, float *total, int *started)
{
    const float part = qr_lane_fold(p);
    *total = *started ? *total + part : part;
    *started = 1;
    memset(p, 0, 32 * sizeof(float));
}

/* Starts a new segment at `row` (rows counted from the panel start k). */
#define QR_SEG_EDGE(row, first, k, seg) ((seg) && (row) > (first) && ((row) - (k)) % (seg) == 0)

/* Segmented lane sum over rows [first, m) of x[row] * y[row]. */
static float qr_seg_dot(int m, int k, int seg, int first, const float *x, const float *y)
{
    float p[32] = {0}, total = 0.0f;
    int started = 0;
    for (int row = first; row < m; ++row)
    {
        if (QR_SEG_EDGE(row, first, k, seg)) qr_seg_flush(p, &total, &started);
        p[row & 31] = fmaf(x[row], y[row], p[row & 31]);
    }
    qr_seg_flush(p, &total, &started);
    return total;
}

/* Factor panel columns [k, k+kb) of rows [k, m).  Per column c every reduction over the rows
 * below c is taken at once from the column as it stands (x = A(c+1:m, c)): sumsq = sum x_i^2
 * and, for each later panel column j, S_j = sum x_i A(i, j).  Then LAPACK's beta, tau and
 * scale = 1 / (alpha - beta); v_i = x_i * scale; w_j = tau * fma(scale, S_j, A(c, j)), which is
 * tau v^T a_j with v_c = 1; A(c, j) = fma(-w_j, 1, A(c, j)) and A(i, j) = fma(-w_j, v_i, A(i, j)). */
static void qr_panel(int m, int k, int kb, float *a, int lda, float *tau)
{
    const int seg = qr_panel_seg(m - k, kb, 50 * 1024);
    float S[QR_NB];
    for (int c = k; c < k + kb; ++c)
    {
        float *x = a + (int64_t)c * lda;
        tau[c] = 0.0f;
        if (m - c <= 1) continue;
        const float sumsq = qr_seg_dot(m, k, seg, c + 1, x, x);
        for (int j = c + 1; j < k + kb; ++j) S[j - c] = qr_seg_dot(m, k, seg, c + 1, x, a + (int64_t)j * lda);
        if (sumsq == 0.0f) continue;
        const float alpha = x[c];
        const float norm = sqrtf(alpha * alpha + sumsq);
        const float beta = alpha >= 0.0f ? -norm : norm;
        const float t = (beta - alpha) / beta;
        const float scale = 1.0f / (alpha - beta);
        tau[c] = t;
        for (int j = c + 1; j < k + kb; ++j)
        {
            float *y = a + (int64_t)j * lda;
            const float w = t * fmaf(scale, S[j - c], y[c]);
            y[c] = fmaf(-w, 1.0f, y[c]);
            for (int row = c + 1; row < m; ++row) y[row] = fmaf(-w, x[row] * scale, y[row]);
        }
        for (int row = c + 1; row < m; ++row) x[row] = x[row] * scale;
        x[c] = beta;
    }
}

/* T (kb x kb, upper, ld 32) of the panel's reflectors (slarft, forward, columnwise). */
static void qr_larft(int m, int k, int kb, const float *a, int lda, const float *tau, float *T)
{
    float d[QR_NB];
    for (int i = 0; i < kb; ++i)
    {
        const float ti = tau[k + i];
        if (ti == 0.0f)
        {
            for (int r = 0; r <= i; ++r) T[i * QR_NB + r] = 0.0f;
            continue;
        }
        for (int r = 0; r < i; ++r)
        {
            float p[32] = {0};
            for (int row = k + i; row < m; ++row)
                p[row & 31] = fmaf(RAT(a, lda, row, k + r), qr_v(a, lda, k, i, row), p[row & 31]);
            d[r] = (-ti) * qr_lane_fold(p);
        }
        for (int r = 0; r < i; ++r)
        {
            float acc = 0.0f;
            for (int q = r; q < i; ++q) acc = fmaf(T[q * QR_NB + r], d[q], acc);
            T[i * QR_NB + r] = acc;
        }
        T[i * QR_NB + i] = ti;
    }
}

/* Columns [0, ncols) of C (rows [k, m), ld ldc): C = (I - V op(T) V^T) C with op(T) = T^T when
 * tr, else T.  V = the panel at columns [k, k+kb) of a. */
static void qr_apply_left(int m, int k, int kb, const float *a, int lda, const float *T, int tr, float *c,
                          int ldc, int ncols)
{
    for (int j = 0; j < ncols; ++j)
    {
        float w[QR_NB], w2[QR_NB];
        for (int i = 0; i < kb; ++i)
        {
            float p[32] = {0};
            for (int row = k + i; row < m; ++row)
                p[row & 31] = fmaf(qr_v(a, lda, k, i, row), RAT(c, ldc, row, j), p[row & 31]);
            w[i] = qr_lane_fold(p);
        }
        for (int i = 0; i < kb; ++i)
        {
            float acc = 0.0f;
            if (tr)
                for (int q = 0; q <= i; ++q) acc = fmaf(T[i * QR_NB + q], w[q], acc);
            else
                for (int q = i; q < kb; ++q) acc = fmaf(T[q * QR_NB + i], w[q], acc);
            w2[i] = acc;
        }
        for (int row = k; row < m; ++row)
        {
            float x = RAT(c, ldc, row, j);
            for (int i = 0; i < kb && i <= row - k; ++i) x = fmaf(-qr_v(a, lda, k, i, row), w2[i], x);
            RAT(c, ldc, row, j) = x;
        }
    }
}

/* Rows [0, nrows) of C (columns [k, nq), ld ldc): C = C (I - V op(T) V^T), op(T) = T when
 * !tr (C Q), T^T when tr (C Q^T). */
static void qr_apply_right(int nq, int k, int kb, const float *a, int lda, const float *T, int tr, float *c,
                           int ldc, int nrows)
{
    for (int r = 0; r < nrows; ++r)
    {
        float y[QR_NB], y2[QR_NB];
        for (int i = 0; i < kb; ++i)
        {
            float p[32] = {0};
            for (int col = k + i; col < nq; ++col)
                p[col & 31] = fmaf(qr_v(a, lda, k, i, col), RAT(c, ldc, r, col), p[col & 31]);
            y[i] = qr_lane_fold(p);
        }
        for (int i = 0; i < kb; ++i)
        {
            float acc = 0.0f;
            if (!tr)
                for (int q = 0; q <= i; ++q) acc = fmaf(T[i * QR_NB + q], y[q], acc);
            else
                for (int q = i; q < kb; ++q) acc = fmaf(T[q * QR_NB + i], y[q], acc);
            y2[i] = acc;
        }
        for (int col = k; col < nq; ++col)
        {
            float x = RAT(c, ldc, r, col);
            for (int i = 0; i < kb && i <= col - k; ++i) x = fmaf(-qr_v(a, lda, k, i, col), y2[i], x);
            RAT(c, ldc, r, col) = x;
        }
    }
}

void orc_sgeqrf(int m, int n, float *a, int lda, float *tau)
{
    const int lim = m < n ? m : n;
    float T[QR_NB * QR_NB];
    for (int k = 0; k < lim; k += QR_NB)
    {
        const int kb = lim - k < QR_NB ? lim - k : QR_NB;
        qr_panel(m, k, kb, a, lda, tau);
        if (k + kb < n)
        {
            qr_larft(m, k, kb, a, lda, tau, T);
            qr_apply_left(m, k, kb, a, lda, T, 1, a + (int64_t)(k + kb) * lda, lda, n - k - kb);
        }
    }
}

/* side 0 left (C is m x n, nq = m), 1 right (nq = n); trans 0 applies Q, else Q^T. */
void orc_sormqr(int side, int trans, int m, int n, int k, const float *a, int lda, const float *tau, float *c,
                int ldc)
{
    const int nq = side == 0 ? m : n;
    float T[QR_NB * QR_NB];
    const int npan = (k + QR_NB - 1) / QR_NB;
    /* forward panel order for Q^T from the left and Q from the right */
    const int forward = (side == 0) == (trans != 0);
    for (int s = 0; s < npan; ++s)
    {
        const int pi = forward ? s : npan - 1 - s;
        const int k0 = pi * QR_NB, kb = k - k0 < QR_NB ? k - k0 : QR_NB;
        qr_larft(nq, k0, kb, a, lda, tau, T);
        if (side == 0)
            qr_apply_left(m, k0, kb, a, lda, T, trans != 0, c, ldc, n);
        else
            qr_apply_right(n, k0, kb, a, lda, T, trans != 0, c, ldc, m);
    }
}

/* Q (m x n) from k reflectors in a, overwriting a (the reflectors are copied first). */
void orc_sorgqr(int m, int n, int k, float *a, int lda, const float *tau)
{
    float *v = (float *)malloc(sizeof(float) * (size_t)(m > 0 ? m : 1) * (size_t)(k > 0 ? k : 1));
    for (int j = 0; j < k; ++j)
        for (int r = 0; r < m; ++r) v[(int64_t)j * m + r] = RAT(a, lda, r, j);
    for (int j = 0; j < n; ++j)
        for (int r = 0; r < m; ++r) RAT(a, lda, r, j) = r == j ? 1.0f : 0.0f;
    orc_sormqr(0, 0, m, n, k, v, m, tau, a, lda);
    free(v);
}

/* Least squares, m >= n: X (n x nrhs) from the QR of a (overwritten) and B (read only). */
void orc_sgels(int m, int n, int nrhs, float *a, int lda, const float *b, int ldb, float *x, int ldx, float *tau)
{
    float *y = (float *)malloc(sizeof(float) * (size_t)(m > 0 ? m : 1) * (size_t)(nrhs > 0 ? nrhs : 1));
    for (int j = 0; j < nrhs; ++j)
        for (int r = 0; r < m; ++r) y[(int64_t)j * m + r] = RAT(b, ldb, r, j);
    orc_sgeqrf(m, n, a, lda, tau);
    orc_sormqr(0, 1, m, nrhs, n, a, lda, tau, y, m);
    for (int j = 0; j < nrhs; ++j)
    {
        float *yj = y + (int64_t)j * m;
        for (int p = n - 1; p >= 0; --p)
        {
            yj[p] = yj[p] / RAT(a, lda, p, p);
            for (int i = 0; i < p; ++i) yj[i] = fmaf(-RAT(a, lda, i, p), yj[p], yj[i]);
        }
        for (int r = 0; r < n; ++r) RAT(x, ldx, r, j) = yj[r];
    }
    free(y);
}

/* The reference's CPU golden (QrCore::Geqr2, householder.hpp:144-170, with Larfg :55-141 on
 * its normal path): unblocked, sequential sums.  Used to pin the judges' CPU ratios. */
void orc_sgeqr2_golden(int m, int n, float *a, int lda, float *tau)
{
    const int kmax = m < n ? m : n;
    for (int j = 0; j < kmax; ++j)
    {
        const int len = m - j;
        tau[j] = 0.0f;
        if (len > 1)
        {
            float sumsq = 0.0f;
            for (int i = j + 1; i < m; ++i) sumsq += RAT(a, lda, i, j) * RAT(a, lda, i, j);
            if (sumsq != 0.0f)
            {
                const float al = RAT(a, lda, j, j);
                const float norm = sqrtf(al * al + sumsq);
                const float beta = al >= 0.0f ? -norm : norm;
                tau[j] = (beta - al) / beta;
                const float scale = 1.0f / (al - beta);
                for (int i = j + 1; i < m; ++i) RAT(a, lda, i, j) *= scale;
                RAT(a, lda, j, j) = beta;
            }
        }
        if (tau[j] != 0.0f && j + 1 < n)
        {
            const float beta = RAT(a, lda, j, j);
            RAT(a, lda, j, j) = 1.0f;
            for (int c = j + 1; c < n; ++c)
            {
                float dot = 0.0f;
                for (int r = j; r < m; ++r) dot += RAT(a, lda, r, j) * RAT(a, lda, r, c);
                const float w = tau[j] * dot;
                for (int r = j; r < m; ++r) RAT(a, lda, r, c) -= w * RAT(a, lda, r, j);
            }
            RAT(a, lda, j, j) = beta;
        }
    }
}

/* Block reflector factor T (k x k, ld ldt) of k reflectors in V (n x k, ld ldv), columnwise
 * (slarft).  direct 0 (forward): v_i has its unit at row i and entries below, T upper;
 * direct 1 (backward): the unit at row n-k+i and entries above, T lower.  Each reflector
 * product is a lane sum over its rows; T's column i is -tau_i times the products, carried
 * through the finished part of T by FMA chains (ascending q).  Only the referenced triangle
 * of T is written. */
void orc_slarft(int direct, int n, int k, const float *v, int ldv, const float *tau, float *t, int ldt)
{
    float *g = (float *)malloc(sizeof(float) * (size_t)(k > 0 ? k : 1));
    if (direct == 0)
    {
        for (int i = 0; i < k; ++i)
        {
            const float ti = tau[i];
            if (ti == 0.0f)
            {
                for (int r = 0; r <= i; ++r) RAT(t, ldt, r, i) = 0.0f;
                continue;
            }
            for (int r = 0; r < i; ++r)
            {
                float p[32] = {0};
                for (int row = i; row < n; ++row)
                    p[row & 31] = fmaf(RAT(v, ldv, row, r), row == i ? 1.0f : RAT(v, ldv, row, i), p[row & 31]);
                g[r] = (-ti) * qr_lane_fold(p);
            }
            for (int r = 0; r < i; ++r)
            {
                float acc = 0.0f;
                for (int q = r; q < i; ++q) acc = fmaf(RAT(t, ldt, r, q), g[q], acc);
                RAT(t, ldt, r, i) = acc;
            }
            RAT(t, ldt, i, i) = ti;
        }
    }
    else
    {
        for (int i = k - 1; i >= 0; --i)
        {
            const float ti = tau[i];
            const int unit = n - k + i;
            if (ti == 0.0f)
            {
                for (int r = i; r < k; ++r) RAT(t, ldt, r, i) = 0.0f;
                continue;
            }
            for (int r = i + 1; r < k; ++r)
            {
                float p[32] = {0};
                for (int row = 0; row <= unit; ++row)
                    p[row & 31] = fmaf(RAT(v, ldv, row, r), row == unit ? 1.0f : RAT(v, ldv, row, i), p[row & 31]);
                g[r] = (-ti) * qr_lane_fold(p);
            }
            for (int r = i + 1; r < k; ++r)
            {
                float acc = 0.0f;
                for (int q = i + 1; q <= r; ++q) acc = fmaf(RAT(t, ldt, r, q), g[q], acc);
                RAT(t, ldt, r, i) = acc;
            }
            RAT(t, ldt, i, i) = ti;
        }
    }
    free(g);
}

/* ---------------------------------------------------------------------------------------
 * Complex QR family (complex64 interleaved, column-major)
 *
 * Reflectors follow LAPACK clarfg, as the reference's kernel does
 * (src/cgeqrf/arch35/cgeqrf_reflector_simd.h:89-170): beta = -copysign(||(alpha; x)||, Re alpha),
 * tau = ((beta - Re alpha) / beta, -(Im alpha / beta)), v = x / (alpha - beta), tau = 0 when
 * x is zero and alpha real; Q = H(1)...H(k), H = I - tau v v^H, R = Q^H A.  The schedule and
 * reductions are the real family's (lane sums over rows, 32-column panels, slarft's T, block
 * application), with these complex forms, each an explicit FMA sequence:
 *   conj-dot   acc += conj(v) a : re = fma(v.im, a.im, fma(v.re, a.re, re)),
 *                                 im = fma(-v.im, a.re, fma(v.re, a.im, im))
 *   dot        acc += c v       : re = fma(-c.im, v.im, fma(c.re, v.re, re)),
 *                                 im = fma(c.im, v.re, fma(c.re, v.im, im))
 *   submul     x - a b          (the LU family's SubMul)
 *   submulc    x - y conj(v)    : re = fma(-y.im, v.im, fma(-y.re, v.re, x.re)),
 *                                 im = fma(y.re, v.im, fma(-y.im, v.re, x.im))
 *   mul        a b              : (fma(-a.im, b.im, a.re b.re), fma(a.im, b.re, a.re b.im))
 *   mulc       conj(a) b        : (fma(a.im, b.im, a.re b.re), fma(-a.im, b.re, a.re b.im))
 * The least-squares triangle has a real diagonal, so x_p is divided componentwise by R_pp.
 * ------------------------------------------------------------------------------------- */

static inline cfl q_conjdot(cfl acc, cfl v, cfl a)
{
    cfl r = {fmaf(v.im, a.im, fmaf(v.re, a.re, acc.re)), fmaf(-v.im, a.re, fmaf(v.re, a.im, acc.im))};
    return r;
}
static inline cfl q_dot(cfl acc, cfl c, cfl v)
{
    cfl r = {fmaf(-c.im, v.im, fmaf(c.re, v.re, acc.re)), fmaf(c.im, v.re, fmaf(c.re, v.im, acc.im))};
    return r;
}
static inline cfl q_submulc(cfl x, cfl y, cfl v)
{
    cfl r = {fmaf(-y.im, v.im, fmaf(-y.re, v.re, x.re)), fmaf(y.re, v.im, fmaf(-y.im, v.re, x.im))};
    return r;
}
static inline cfl q_mul(cfl a, cfl b)
{
    cfl r = {fmaf(-a.im, b.im, a.re * b.re), fmaf(a.im, b.re, a.re * b.im)};
    return r;
}
static inline cfl q_mulc(cfl a, cfl b)
{
    cfl r = {fmaf(a.im, b.im, a.re * b.re), fmaf(-a.im, b.re, a.re * b.im)};
    return r;
}
static inline cfl q_fma(cfl a, cfl b, cfl acc) /* acc + a b */
{
    cfl r = {fmaf(-a.im, b.im, fmaf(a.re, b.re, acc.re)), fmaf(a.im, b.re, fmaf(a.re, b.im, acc.im))};
    return r;
}
static inline cfl q_fmac(cfl a, cfl b, cfl acc) /* acc + conj(a) b */
{
    cfl r = {fmaf(a.im, b.im, fmaf(a.re, b.re, acc.re)), fmaf(-a.im, b.re, fmaf(a.re, b.im, acc.im))};
    return r;
}

static cfl q_fold(cfl *p)
{
    float re[32], im[32];
    for (int l = 0; l < 32; ++l)
    {
        re[l] = p[l].re;
        im[l] = p[l].im;
    }
    cfl r = {qr_lane_fold(re), qr_lane_fold(im)};
    return r;
}

static inline cfl cq_v(const cfl *a, int lda, int k, int i, int row)
{
    if (row == k + i)
    {
        cfl one = {1.0f, 0.0f};
        return one;
    }
    return CAT(a, lda, row, k + i);
}

static void cq_seg_flush(cfl *p, cfl *total, int *started)
{
    const cfl part = q_fold(p);
    if (*started)
    {
        total->re = total->re + part.re;
        total->im = total->im + part.im;
    }
    else
        *total = part;
    *started = 1;
    memset(p, 0, 32 * sizeof(cfl));
}

/* Segmented lane sums over rows [first, m): of |x_i|^2, and of conj(x_i) y_i. */
static float cq_seg_sumsq(int m, int k, int seg, int first, const cfl *x)
{
    float p[32] = {0}, total = 0.0f;
    int started = 0;
    for (int row = first; row < m; ++row)
    {
        if (QR_SEG_EDGE(row, first, k, seg)) qr_seg_flush(p, &total, &started);
        p[row & 31] = fmaf(x[row].im, x[row].im, fmaf(x[row].re, x[row].re, p[row & 31]));
    }
    qr_seg_flush(p, &total, &started);
    return total;
}

static cfl cq_seg_conjdot(int m, int k, int seg, int first, const cfl *x, const cfl *y)
{
    cfl p[32], total = {0.0f, 0.0f};
    int started = 0;
    memset(p, 0, sizeof p);
    for (int row = first; row < m; ++row)
    {
        if (QR_SEG_EDGE(row, first, k, seg)) cq_seg_flush(p, &total, &started);
        p[row & 31] = q_conjdot(p[row & 31], x[row], y[row]);
    }
    cq_seg_flush(p, &total, &started);
    return total;
}

/* Panels are reduced in segments as in the real family (qr_panel_seg, a budget of 25,600
 * complex elements per block) and, as there, every reduction of column c's step is taken at
 * once from the column as it stands (x = A(c+1:m, c)): sumsq = sum |x_i|^2 and, per later panel
 * column j, S_j = sum conj(x_i) A(i, j).  With d = alpha - beta = (dr, di), den = |d|^2 and
 * g = (dr / den, di / den): v_i = x_i / d (two real divisions per part), v^H a_j =
 * A(c, j) + g S_j (one complex FMA sequence), w_j = conj(tau) v^H a_j. */
static void cq_panel(int m, int k, int kb, cfl *a, int lda, cfl *tau)
{
    const int seg = qr_panel_seg(m - k, kb, 25 * 1024);
    cfl S[QR_NB];
    const cfl one = {1.0f, 0.0f};
    for (int c = k; c < k + kb; ++c)
    {
        cfl *x = a + (int64_t)c * lda;
        tau[c].re = tau[c].im = 0.0f;
        const float sumsq = cq_seg_sumsq(m, k, seg, c + 1, x);
        for (int j = c + 1; j < k + kb; ++j) S[j - c] = cq_seg_conjdot(m, k, seg, c + 1, x, a + (int64_t)j * lda);
        const cfl al = x[c];
        if (sumsq == 0.0f && al.im == 0.0f) continue;
        const float norm = sqrtf(al.re * al.re + al.im * al.im + sumsq);
        const float beta = copysignf(norm, al.re) * -1.0f;
        const cfl t = {(beta - al.re) / beta, -(al.im / beta)};
        const float dr = al.re - beta, di = al.im;
        const float den = dr * dr + di * di;
        const cfl g = {dr / den, di / den};
        tau[c] = t;
        for (int j = c + 1; j < k + kb; ++j)
        {
            cfl *y = a + (int64_t)j * lda;
            const cfl w = q_mulc(t, q_fma(g, S[j - c], y[c]));
            y[c] = c_submul(y[c], one, w);
            for (int row = c + 1; row < m; ++row)
            {
                const cfl v = {(x[row].re * dr + x[row].im * di) / den, (x[row].im * dr - x[row].re * di) / den};
                y[row] = c_submul(y[row], v, w);
            }
        }
        for (int row = c + 1; row < m; ++row)
        {
            const cfl v = {(x[row].re * dr + x[row].im * di) / den, (x[row].im * dr - x[row].re * di) / den};
            x[row] = v;
        }
        x[c].re = beta;
        x[c].im = 0.0f;
    }
}

/* T (kb x kb upper, ld 32) of the panel's reflectors: T(i,i) = tau_i, T(0:i, i) = T(0:i, 0:i) d,
 * d_r = -tau_i (v_r^H v_i). */
static void cq_larft(int nq, int k, int kb, const cfl *a, int lda, const cfl *tau, cfl *T)
{
    cfl d[QR_NB];
    for (int i = 0; i < kb; ++i)
    {
        const cfl ti = tau[k + i];
        if (ti.re == 0.0f && ti.im == 0.0f)
        {
            for (int r = 0; r <= i; ++r) T[i * QR_NB + r] = (cfl){0.0f, 0.0f};
            continue;
        }
        const cfl nt = {-ti.re, -ti.im};
        for (int r = 0; r < i; ++r)
        {
            cfl p[32];
            memset(p, 0, sizeof p);
            for (int row = k + i; row < nq; ++row)
                p[row & 31] = q_conjdot(p[row & 31], CAT(a, lda, row, k + r), cq_v(a, lda, k, i, row));
            d[r] = q_mul(nt, q_fold(p));
        }
        for (int r = 0; r < i; ++r)
        {
            cfl acc = {0.0f, 0.0f};
            for (int q = r; q < i; ++q) acc = q_fma(T[q * QR_NB + r], d[q], acc);
            T[i * QR_NB + r] = acc;
        }
        T[i * QR_NB + i] = ti;
    }
}

/* Left: C = (I - V op(T) V^H) C, op(T) = T^H when herm (Q^H C), T otherwise (Q C). */
static void cq_apply_left(int m, int k, int kb, const cfl *a, int lda, const cfl *T, int herm, cfl *c, int ldc,
                          int ncols)
{
    for (int j = 0; j < ncols; ++j)
    {
        cfl w[QR_NB], w2[QR_NB];
        for (int i = 0; i < kb; ++i)
        {
            cfl p[32];
            memset(p, 0, sizeof p);
            for (int row = k + i; row < m; ++row)
                p[row & 31] = q_conjdot(p[row & 31], cq_v(a, lda, k, i, row), CAT(c, ldc, row, j));
            w[i] = q_fold(p);
        }
        for (int i = 0; i < kb; ++i)
        {
            cfl acc = {0.0f, 0.0f};
            if (herm)
                for (int q = 0; q <= i; ++q) acc = q_fmac(T[i * QR_NB + q], w[q], acc);
            else
                for (int q = i; q < kb; ++q) acc = q_fma(T[q * QR_NB + i], w[q], acc);
            w2[i] = acc;
        }
        for (int row = k; row < m; ++row)
        {
            cfl x = CAT(c, ldc, row, j);
            for (int i = 0; i < kb && i <= row - k; ++i) x = c_submul(x, cq_v(a, lda, k, i, row), w2[i]);
            CAT(c, ldc, row, j) = x;
        }
    }
}

/* Right: C = C (I - V op(T) V^H), op(T) = T (C Q) or T^H when herm (C Q^H). */
static void cq_apply_right(int nq, int k, int kb, const cfl *a, int lda, const cfl *T, int herm, cfl *c, int ldc,
                           int nrows)
{
    for (int r = 0; r < nrows; ++r)
    {
        cfl y[QR_NB], y2[QR_NB];
        for (int i = 0; i < kb; ++i)
        {
            cfl p[32];
            memset(p, 0, sizeof p);
            for (int col = k + i; col < nq; ++col)
                p[col & 31] = q_dot(p[col & 31], CAT(c, ldc, r, col), cq_v(a, lda, k, i, col));
            y[i] = q_fold(p);
        }
        for (int i = 0; i < kb; ++i)
        {
            cfl acc = {0.0f, 0.0f};
            if (!herm)
                for (int q = 0; q <= i; ++q) acc = q_fma(T[i * QR_NB + q], y[q], acc);
            else
                for (int q = i; q < kb; ++q) acc = q_fmac(T[q * QR_NB + i], y[q], acc);
            y2[i] = acc;
        }
        for (int col = k; col < nq; ++col)
        {
            cfl x = CAT(c, ldc, r, col);
            for (int i = 0; i < kb && i <= col - k; ++i) x = q_submulc(x, y2[i], cq_v(a, lda, k, i, col));
            CAT(c, ldc, r, col) = x;
        }
    }
}

void orc_cgeqrf(int m, int n, float *af, int lda, float *tauf)
{
    cfl *a = (cfl *)af, *tau = (cfl *)tauf;
    const int lim = m < n ? m : n;
    cfl T[QR_NB * QR_NB];
    for (int k = 0; k < lim; k += QR_NB)
    {
        const int kb = lim - k < QR_NB ? lim - k : QR_NB;
        cq_panel(m, k, kb, a, lda, tau);
        if (k + kb < n)
        {
            cq_larft(m, k, kb, a, lda, tau, T);
            cq_apply_left(m, k, kb, a, lda, T, 1, a + (int64_t)(k + kb) * lda, lda, n - k - kb);
        }
    }
}

/* side 0 left (nq = m), 1 right (nq = n); herm 0 applies Q, 1 applies Q^H. */
void orc_cunmqr(int side, int herm, int m, int n, int k, const float *af, int lda, const float *tauf, float *cf,
                int ldc)
{
    const cfl *a = (const cfl *)af, *tau = (const cfl *)tauf;
    cfl *c = (cfl *)cf;
    const int nq = side == 0 ? m : n;
    cfl T[QR_NB * QR_NB];
    const int npan = (k + QR_NB - 1) / QR_NB;
    const int forward = (side == 0) == (herm != 0);
    for (int s = 0; s < npan; ++s)
    {
        const int pi = forward ? s : npan - 1 - s;
        const int k0 = pi * QR_NB, kb = k - k0 < QR_NB ? k - k0 : QR_NB;
        cq_larft(nq, k0, kb, a, lda, tau, T);
        if (side == 0)
            cq_apply_left(m, k0, kb, a, lda, T, herm, c, ldc, n);
        else
            cq_apply_right(n, k0, kb, a, lda, T, herm, c, ldc, m);
    }
}

void orc_cungqr(int m, int n, int k, float *af, int lda, const float *tauf)
{
    cfl *a = (cfl *)af;
    cfl *v = (cfl *)malloc(sizeof(cfl) * (size_t)(m > 0 ? m : 1) * (size_t)(k > 0 ? k : 1));
    for (int j = 0; j < k; ++j)
        for (int r = 0; r < m; ++r) v[(int64_t)j * m + r] = CAT(a, lda, r, j);
    for (int j = 0; j < n; ++j)
        for (int r = 0; r < m; ++r) CAT(a, lda, r, j) = (cfl){r == j ? 1.0f : 0.0f, 0.0f};
    orc_cunmqr(0, 0, m, n, k, (const float *)v, m, tauf, af, lda);
    free(v);
}

/* Returns the one-based position of the first zero diagonal entry of R (X then untouched),
 * as the reference's back substitution reports it (src/ccgels/arch35/ccgels_kernel.cpp:150-176,
 * FindZeroDiagonal), else 0. */
int orc_cgels(int m, int n, int nrhs, float *af, int lda, const float *bf, int ldb, float *xf, int ldx, float *tauf)
{
    cfl *a = (cfl *)af, *x = (cfl *)xf;
    const cfl *b = (const cfl *)bf;
    cfl *y = (cfl *)malloc(sizeof(cfl) * (size_t)(m > 0 ? m : 1) * (size_t)(nrhs > 0 ? nrhs : 1));
    for (int j = 0; j < nrhs; ++j)
        for (int r = 0; r < m; ++r) y[(int64_t)j * m + r] = CAT(b, ldb, r, j);
    orc_cgeqrf(m, n, af, lda, tauf);
    orc_cunmqr(0, 1, m, nrhs, n, af, lda, tauf, (float *)y, m);
    for (int p = 0; p < n; ++p)
        if (CAT(a, lda, p, p).re == 0.0f && CAT(a, lda, p, p).im == 0.0f)
        {
            free(y);
            return p + 1;
        }
    for (int j = 0; j < nrhs; ++j)
    {
        cfl *yj = y + (int64_t)j * m;
        for (int p = n - 1; p >= 0; --p)
        {
            const float d = CAT(a, lda, p, p).re;
            yj[p].re = yj[p].re / d;
            yj[p].im = yj[p].im / d;
            for (int i = 0; i < p; ++i) yj[i] = c_submul(yj[i], CAT(a, lda, i, p), yj[p]);
        }
        for (int r = 0; r < n; ++r) CAT(x, ldx, r, j) = yj[r];
    }
    free(y);
    return 0;
}
