/*
 * lapack_host.c -- the host LAPACK the reference's tests use as their golden, driven over
 * whole batches for the benchmark's CPU baseline.
 *
 * BENCHMARK AND TEST INFRASTRUCTURE ONLY.  The library (libops_solver.so) never links,
 * loads or calls it.
 *
 * The reference judges its device results against scipy's FP32 LAPACK
 * (test/cholesky/lapack_residual.py:64-86 calls scipy.linalg.lapack.spotrf/spotrs;
 * test/utils/cholesky/fixtures.py:108-136 calls cpotrf/cpotrs; the LU tests use
 * sgetrf/sgetrs/sgetri).  scipy bundles OpenBLAS as libscipy_openblas*.so and exports the
 * LAPACKE C interface with a scipy_ prefix.  This file dlopen()s that library (the path is
 * passed in by the caller, resolved from scipy's install) and runs the same routines over a
 * batch: OpenMP over matrices with OpenBLAS held to one thread per call for the batched
 * workloads, OpenBLAS's own threads for one large system.
 *
 * Matrices are column-major.  Every routine first copies its inputs into caller-provided
 * work buffers (LAPACK factors in place), so repeated passes over the same inputs do the
 * same work.
 */
#include <dlfcn.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define COL_MAJOR 102

typedef int (*getrf_t)(int, int, int, float *, int, int *);
typedef int (*getrs_t)(int, char, int, int, const float *, int, const int *, float *, int);
typedef int (*getri_t)(int, int, float *, int, const int *);
typedef int (*potrf_t)(int, char, int, float *, int);
typedef int (*potrs_t)(int, char, int, int, const float *, int, float *, int);
/* complex64 is passed as interleaved float pairs (lapack_complex_float is layout-equal) */
typedef int (*cpotrf_t)(int, char, int, void *, int);
typedef int (*cpotrs_t)(int, char, int, int, const void *, int, void *, int);
typedef void (*set_threads_t)(int);
typedef char *(*get_config_t)(void);

static void *lib;
static getrf_t sgetrf;
static getrs_t sgetrs;
static getri_t sgetri;
static potrf_t spotrf;
static potrs_t spotrs;
static cpotrf_t cpotrf;
static cpotrs_t cpotrs;
static set_threads_t set_threads;
static get_config_t get_config;

/* Loads the OpenBLAS library at `path`; 0 on success, -1 when a symbol is missing. */
int lh_open(const char *path)
{
    if (lib) return 0;
    lib = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!lib) return -1;
    sgetrf = (getrf_t)dlsym(lib, "scipy_LAPACKE_sgetrf");
    sgetrs = (getrs_t)dlsym(lib, "scipy_LAPACKE_sgetrs");
    sgetri = (getri_t)dlsym(lib, "scipy_LAPACKE_sgetri");
    spotrf = (potrf_t)dlsym(lib, "scipy_LAPACKE_spotrf");
    spotrs = (potrs_t)dlsym(lib, "scipy_LAPACKE_spotrs");
    cpotrf = (cpotrf_t)dlsym(lib, "scipy_LAPACKE_cpotrf");
    cpotrs = (cpotrs_t)dlsym(lib, "scipy_LAPACKE_cpotrs");
    set_threads = (set_threads_t)dlsym(lib, "scipy_openblas_set_num_threads");
    get_config = (get_config_t)dlsym(lib, "scipy_openblas_get_config");
    if (!sgetrf || !sgetrs || !sgetri || !spotrf || !spotrs || !cpotrf || !cpotrs || !set_threads) return -1;
    return 0;
}

const char *lh_config(void) { return get_config ? get_config() : "unknown"; }

int lh_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void lh_blas_threads(int n) { set_threads(n); }

/* Config 1 shape: spotrf (lower or upper) then spotrs, `count` matrices of order n with
 * nrhs right-hand sides each; a, b pristine inputs; w, x outputs (factor, solution). */
void lh_potrf_potrs_batched(int n, int nrhs, int upper, const float *a, float *w, const float *b, float *x,
                            int count, int *info, int threads)
{
    const char uplo = upper ? 'U' : 'L';
    set_threads(1);
#pragma omp parallel for schedule(static) num_threads(threads)
    for (int q = 0; q < count; ++q)
    {
        const int64_t sa = (int64_t)n * n, sb = (int64_t)n * nrhs;
        memcpy(w + q * sa, a + q * sa, sizeof(float) * sa);
        memcpy(x + q * sb, b + q * sb, sizeof(float) * sb);
        int st = spotrf(COL_MAJOR, uplo, n, w + q * sa, n);
        if (st == 0) st = spotrs(COL_MAJOR, uplo, n, nrhs, w + q * sa, n, x + q * sb, n);
        info[q] = st;
    }
}

/* Configs 2 and 4 shape: sgetrf, sgetrs (no transpose), and when `inv` is not NULL the
 * inverse (the factor copied to inv, then sgetri). */
void lh_getrf_getrs_batched(int n, int nrhs, const float *a, float *w, const float *b, float *x, float *inv,
                            int *ipiv, int count, int *info, int threads)
{
    set_threads(1);
#pragma omp parallel for schedule(static) num_threads(threads)
    for (int q = 0; q < count; ++q)
    {
        const int64_t sa = (int64_t)n * n, sb = (int64_t)n * nrhs;
        float *wq = w + q * sa;
        int *pq = ipiv + (int64_t)q * n;
        memcpy(wq, a + q * sa, sizeof(float) * sa);
        memcpy(x + q * sb, b + q * sb, sizeof(float) * sb);
        int st = sgetrf(COL_MAJOR, n, n, wq, n, pq);
        if (st >= 0) sgetrs(COL_MAJOR, 'N', n, nrhs, wq, n, pq, x + q * sb, n);
        if (inv && st == 0)
        {
            memcpy(inv + q * sa, wq, sizeof(float) * sa);
            st = sgetri(COL_MAJOR, n, inv + q * sa, n, pq);
        }
        info[q] = st;
    }
}

/* Config 3 shape: complex64 cpotrf + cpotrs over matrices of different orders.  Matrix q
 * has order orders[q], leading dimension orders[q], and starts at float offset a_off[q]
 * (b_off[q] for its right-hand sides); the largest orders are handed out first. */
void lh_cpotrf_cpotrs_vbatched(const int *orders, const int64_t *a_off, const int64_t *b_off, const float *a,
                               float *w, const float *b, float *x, int nrhs, int count, int *info, int threads)
{
    set_threads(1);
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads)
    for (int q = 0; q < count; ++q)
    {
        const int n = orders[q];
        const int64_t sa = 2 * (int64_t)n * n, sb = 2 * (int64_t)n * nrhs;
        memcpy(w + a_off[q], a + a_off[q], sizeof(float) * sa);
        memcpy(x + b_off[q], b + b_off[q], sizeof(float) * sb);
        int st = n ? cpotrf(COL_MAJOR, 'L', n, w + a_off[q], n) : 0;
        if (st == 0 && n) st = cpotrs(COL_MAJOR, 'L', n, nrhs, w + a_off[q], n, x + b_off[q], n);
        info[q] = st;
    }
}

/* Config 5 shape: one large system, OpenBLAS threaded (blas_threads), sgetrf + sgetrs. */
int lh_sgesv_single(int n, int nrhs, const float *a, float *w, const float *b, float *x, int *ipiv,
                    int blas_threads)
{
    set_threads(blas_threads);
    memcpy(w, a, sizeof(float) * (int64_t)n * n);
    memcpy(x, b, sizeof(float) * (int64_t)n * nrhs);
    int st = sgetrf(COL_MAJOR, n, n, w, n, ipiv);
    if (st >= 0) sgetrs(COL_MAJOR, 'N', n, nrhs, w, n, ipiv, x, n);
    set_threads(1);
    return st;
}

/* One large SPD matrix: spotrf (lower) with OpenBLAS threaded (blas_threads). */
int lh_spotrf_single(int n, const float *a, float *w, int blas_threads)
{
    set_threads(blas_threads);
    memcpy(w, a, sizeof(float) * (int64_t)n * n);
    int st = spotrf(COL_MAJOR, 'L', n, w, n);
    set_threads(1);
    return st;
}
