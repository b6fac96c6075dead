// api_cqr.cpp -- complex QR family C entry points: Cgeqrf, Cungqr, Cunmqr, CCgels (+ _bufferSize).
//
// Argument ladders and status rules follow the reference host code (paths relative to the
// reference root):
//   shared run  src/utils/complex_qr/arch35/complex_qr_host.cpp:17-160 (ComplexQrQuery / Run:
//               null handle first; shape ladder; the workspace pointer and size; a null info
//               returns INVALID_VALUE; an empty problem writes info 0; then the inputs are
//               screened for NaN / Inf on the device, the stream synchronised and the status
//               read back, INVALID_VALUE with info -i on a non-finite input)
//   Cgeqrf      src/cgeqrf/arch35/cgeqrf_host.cpp:19-77 (1 m, 2 n, 3 A, 4 lda, 5 TAU,
//               6 Workspace, 7 Lwork; screens A -> 3)
//   Cungqr      src/cungqr/arch35/cungqr_host.cpp:19-85 (1 m, 2 n (n > m), 3 k (k > n), 4 A,
//               5 lda, 6 tau, 7 work, 8 lwork; screens the reflectors -> 4, tau -> 6)
//   Cunmqr      src/cunmqr/arch35/cunmqr_host.cpp:29-120 (1 side, 2 trans (N or C), 3 m, 4 n,
//               5 k, 6 A, 7 lda, 8 tau, 9 C, 10 ldc, 11 work, 12 lwork; reflectors -> 6,
//               tau -> 8, C -> 9)
//   CCgels      src/ccgels/arch35/ccgels_host.cpp:22-150 (1 m (m < n), 2 n, 3 nrhs, 4 dA, 5 lda,
//               6 dB, 7 ldb, 8 dX, 9 ldx, then dX overlapping dA or dB -> 8, nrhs > 128 -> 3,
//               m or n > 4096 -> 1; 10 workspace, 11 bytes, 12 niter; screens dA -> 4, dB -> 6)
// Workspace sizes are this build's: one 32 x 32 complex block factor (two for Cgeqrf and CCgels,
// whose look-ahead keeps consecutive panels' factors), plus the reflector copy (Cungqr) or tau
// and Q^H B (CCgels).
#include <limits.h>

#include <algorithm>

#include "handle.h"
#include "launch.h"
#include "launch_qr.h"

using namespace ops_solver;

namespace
{
constexpr int GELS_MAX_DIM = 4096;
constexpr int GELS_MAX_RHS = 128;
constexpr size_t CPLX = sizeof(float2);

bool span_ok(const void *p, size_t bytes)
{
    return p && reinterpret_cast<uintptr_t>(p) % alignof(float) == 0 && is_device_pointer(p) &&
           device_span(p, bytes);
}

bool overlap(const void *a, size_t abytes, const void *b, size_t bbytes)
{
    uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    return x <= y ? y - x < abytes : x - y < bbytes;
}

// -argument into a usable info buffer; INVALID_VALUE.
aclsolverStatus_t bad(Handle *h, int *info, int argument)
{
    if (span_ok(info, sizeof(int)) && launch_fill_info(info, -argument, 1, h->stream) != cudaSuccess)
        cudaGetLastError();
    return ACLSOLVER_STATUS_INVALID_VALUE;
}

aclsolverStatus_t info_zero(Handle *h, int *info) { return launch_status(launch_fill_info(info, 0, 1, h->stream)); }

aclsolverStatus_t finish(cudaError_t e)
{
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        return ACLSOLVER_STATUS_EXECUTION_FAILED;
    }
    return ACLSOLVER_STATUS_SUCCESS;
}

// Screens the regions on the device and reads the verdict back (a stream synchronisation):
// SUCCESS when all are finite, else INVALID_VALUE with info = -(smallest failing code).
aclsolverStatus_t screen(Handle *h, int *info, const CqRegion *regions, int count)
{
    cudaError_t e = launch_fill_info(info, INT_MAX, 1, h->stream);
    if (e == cudaSuccess) e = launch_cq_finite(regions, count, info, h->stream);
    int flag = INT_MAX;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, info, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        return ACLSOLVER_STATUS_EXECUTION_FAILED;
    }
    if (flag != INT_MAX) return bad(h, info, flag);
    return info_zero(h, info);
}

int geqrf_shape(int m, int n, const void *A, int lda)
{
    if (m < 0) return 1;
    if (n < 0) return 2;
    if (m && n && !A) return 3;
    if (lda < std::max(1, m)) return 4;
    return 0;
}

int ungqr_shape(int m, int n, int k, const void *A, int lda, const void *tau)
{
    if (m < 0) return 1;
    if (n < 0 || n > m) return 2;
    if (k < 0 || k > n) return 3;
    if (m && n && !A) return 4;
    if (lda < std::max(1, m)) return 5;
    if (k && !tau) return 6;
    return 0;
}

int unmqr_shape(int side, int trans, int m, int n, int k, const void *A, int lda, const void *tau, const void *C,
                int ldc)
{
    if (side != ACLSOLVER_SIDE_LEFT && side != ACLSOLVER_SIDE_RIGHT) return 1;
    if (trans != ACLSOLVER_OP_N && trans != ACLSOLVER_OP_C) return 2;
    if (m < 0) return 3;
    if (n < 0) return 4;
    const int order = side == ACLSOLVER_SIDE_LEFT ? m : n;
    if (k < 0 || k > order) return 5;
    const bool active = m && n && k;
    if (active && !A) return 6;
    if (lda < std::max(1, order)) return 7;
    if (active && !tau) return 8;
    if (active && !C) return 9;
    if (ldc < std::max(1, m)) return 10;
    return 0;
}

int gels_shape(int m, int n, int nrhs, const void *A, int lda, const void *B, int ldb, const void *X, int ldx)
{
    if (m < 0 || m < n) return 1;
    if (n < 0) return 2;
    if (nrhs < 0) return 3;
    const bool active = m && n && nrhs;
    if (active && !A) return 4;
    if (lda < std::max(1, m)) return 5;
    if (active && !B) return 6;
    if (ldb < std::max(1, m)) return 7;
    if (active && !X) return 8;
    if (ldx < std::max(1, n)) return 9;
    if (!active) return 0;
    const size_t xb = (size_t)nrhs * ldx * CPLX;
    if (overlap(X, xb, A, (size_t)n * lda * CPLX) || overlap(X, xb, B, (size_t)nrhs * ldb * CPLX)) return 8;
    if (nrhs > GELS_MAX_RHS) return 3;
    if (m > GELS_MAX_DIM || n > GELS_MAX_DIM) return 1;
    return 0;
}

size_t ungqr_elems(int m, int n, int k) { return m == 0 || n == 0 ? 0 : (size_t)m * k + QR_T_FLOATS; }

bool as_count(size_t elems, int *out)
{
    if (elems > (size_t)INT_MAX) return false;
    *out = (int)elems;
    return true;
}
}  // namespace

extern "C"
{
    aclsolverStatus_t aclsolverCgeqrf_bufferSize(aclsolverHandle_t handle, int m, int n, aclsolverFloatComplex *A,
                                                 int lda, int *Lwork)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        if (!Lwork || geqrf_shape(m, n, A, lda)) return ACLSOLVER_STATUS_INVALID_VALUE;
        *Lwork = m == 0 || n == 0 ? 0 : QR_GEQRF_T_FLOATS;
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverCgeqrf(aclsolverHandle_t handle, int m, int n, aclsolverFloatComplex *A, int lda,
                                      aclsolverFloatComplex *TAU, aclsolverFloatComplex *Workspace, int Lwork,
                                      int *devInfo)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        const bool empty = m == 0 || n == 0;
        int b = geqrf_shape(m, n, A, lda);
        if (!b && !empty && !TAU) b = 5;
        const int need = empty ? 0 : QR_GEQRF_T_FLOATS;
        if (!b && Lwork < need) b = 7;
        if (!b && need && !Workspace) b = 6;
        if (!devInfo) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (b) return bad(h, devInfo, b);
        if (!span_ok(devInfo, sizeof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (empty) return info_zero(h, devInfo);
        if (!span_ok(A, (size_t)lda * n * CPLX)) return bad(h, devInfo, 3);
        if (!span_ok(TAU, (size_t)std::min(m, n) * CPLX)) return bad(h, devInfo, 5);
        if (!span_ok(Workspace, (size_t)need * CPLX)) return bad(h, devInfo, 6);
        const CqRegion regions[1] = {{A, m, n, lda, 0, 3}};
        aclsolverStatus_t st = screen(h, devInfo, regions, 1);
        if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        return finish(launch_cgeqrf(reinterpret_cast<float2 *>(A), lda, m, n, reinterpret_cast<float2 *>(TAU),
                                    reinterpret_cast<float2 *>(Workspace), h->stream));
    }

    aclsolverStatus_t aclsolverCungqr_bufferSize(aclsolverHandle_t handle, int m, int n, int k,
                                                 const aclsolverFloatComplex *A, int lda,
                                                 const aclsolverFloatComplex *tau, int *lwork)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        if (!lwork || ungqr_shape(m, n, k, A, lda, tau)) return ACLSOLVER_STATUS_INVALID_VALUE;
        return as_count(ungqr_elems(m, n, k), lwork) ? ACLSOLVER_STATUS_SUCCESS : ACLSOLVER_STATUS_INVALID_VALUE;
    }

    aclsolverStatus_t aclsolverCungqr(aclsolverHandle_t handle, int m, int n, int k, aclsolverFloatComplex *A,
                                      int lda, const aclsolverFloatComplex *tau, aclsolverFloatComplex *work,
                                      int lwork, int *devInfo)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        const bool empty = m == 0 || n == 0;
        int b = ungqr_shape(m, n, k, A, lda, tau);
        const size_t need = b ? 0 : ungqr_elems(m, n, k);
        if (!b && (lwork < 0 || (size_t)lwork < need)) b = 8;
        if (!b && need && !work) b = 7;
        if (!devInfo) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (b) return bad(h, devInfo, b);
        if (!span_ok(devInfo, sizeof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (empty) return info_zero(h, devInfo);
        if (!span_ok(A, (size_t)lda * n * CPLX)) return bad(h, devInfo, 4);
        if (k && !span_ok(tau, (size_t)k * CPLX)) return bad(h, devInfo, 6);
        if (!span_ok(work, need * CPLX)) return bad(h, devInfo, 7);
        const CqRegion regions[2] = {{A, m, k, lda, 1, 4}, {tau, k, 1, k, 0, 6}};
        aclsolverStatus_t st = screen(h, devInfo, regions, 2);
        if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        return finish(launch_cungqr(m, n, k, reinterpret_cast<float2 *>(A), lda,
                                    reinterpret_cast<const float2 *>(tau), reinterpret_cast<float2 *>(work),
                                    h->stream));
    }

    aclsolverStatus_t aclsolverCunmqr_bufferSize(aclsolverHandle_t handle, aclsolverSideMode_t side,
                                                 aclsolverOperation_t trans, int m, int n, int k,
                                                 const aclsolverFloatComplex *A, int lda,
                                                 const aclsolverFloatComplex *tau, const aclsolverFloatComplex *C,
                                                 int ldc, int *lwork)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        if (!lwork || unmqr_shape(side, trans, m, n, k, A, lda, tau, C, ldc)) return ACLSOLVER_STATUS_INVALID_VALUE;
        *lwork = m == 0 || n == 0 || k == 0 ? 0 : QR_T_FLOATS;
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverCunmqr(aclsolverHandle_t handle, aclsolverSideMode_t side, aclsolverOperation_t trans,
                                      int m, int n, int k, const aclsolverFloatComplex *A, int lda,
                                      const aclsolverFloatComplex *tau, aclsolverFloatComplex *C, int ldc,
                                      aclsolverFloatComplex *work, int lwork, int *devInfo)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        const bool empty = m == 0 || n == 0 || k == 0;
        int b = unmqr_shape(side, trans, m, n, k, A, lda, tau, C, ldc);
        const int need = empty ? 0 : QR_T_FLOATS;
        if (!b && lwork < need) b = 12;
        if (!b && need && !work) b = 11;
        if (!devInfo) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (b) return bad(h, devInfo, b);
        if (!span_ok(devInfo, sizeof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (empty) return info_zero(h, devInfo);
        const int order = side == ACLSOLVER_SIDE_LEFT ? m : n;
        if (!span_ok(A, (size_t)lda * k * CPLX)) return bad(h, devInfo, 6);
        if (!span_ok(tau, (size_t)k * CPLX)) return bad(h, devInfo, 8);
        if (!span_ok(C, (size_t)ldc * n * CPLX)) return bad(h, devInfo, 9);
        if (!span_ok(work, (size_t)need * CPLX)) return bad(h, devInfo, 11);
        const CqRegion regions[3] = {{A, order, k, lda, 1, 6}, {tau, k, 1, k, 0, 8}, {C, m, n, ldc, 0, 9}};
        aclsolverStatus_t st = screen(h, devInfo, regions, 3);
        if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        return finish(launch_cunmqr(side == ACLSOLVER_SIDE_RIGHT, trans == ACLSOLVER_OP_C, m, n, k,
                                    reinterpret_cast<const float2 *>(A), lda, reinterpret_cast<const float2 *>(tau),
                                    reinterpret_cast<float2 *>(C), ldc, reinterpret_cast<float2 *>(work), h->stream));
    }

    aclsolverStatus_t aclsolverCCgels_bufferSize(aclsolverHandle_t handle, int m, int n, int nrhs,
                                                 aclsolverFloatComplex *dA, int ldda, aclsolverFloatComplex *dB,
                                                 int lddb, aclsolverFloatComplex *dX, int lddx, void *dwork,
                                                 size_t *lwork_bytes)
    {
        (void)dwork;
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        if (!lwork_bytes || gels_shape(m, n, nrhs, dA, ldda, dB, lddb, dX, lddx)) return ACLSOLVER_STATUS_INVALID_VALUE;
        *lwork_bytes = m == 0 || n == 0 || nrhs == 0 ? 0 : cgels_work_elems(m, n, nrhs) * CPLX;
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverCCgels(aclsolverHandle_t handle, int m, int n, int nrhs, aclsolverFloatComplex *dA,
                                      int ldda, aclsolverFloatComplex *dB, int lddb, aclsolverFloatComplex *dX,
                                      int lddx, void *dWorkspace, size_t lwork_bytes, int *niter, int *dinfo)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        const bool empty = m == 0 || n == 0 || nrhs == 0;
        int b = gels_shape(m, n, nrhs, dA, ldda, dB, lddb, dX, lddx);
        const size_t need = b || empty ? 0 : cgels_work_elems(m, n, nrhs) * CPLX;
        if (!b && (lwork_bytes < need || lwork_bytes == SIZE_MAX)) b = 11;
        if (!b && need && !dWorkspace) b = 10;
        if (!b && !niter) b = 12;
        if (!dinfo) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (b) return bad(h, dinfo, b);
        if (!span_ok(dinfo, sizeof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
        *niter = 0;  // a direct QR solve: no refinement iterations
        if (empty) return info_zero(h, dinfo);
        if (!span_ok(dA, (size_t)ldda * n * CPLX)) return bad(h, dinfo, 4);
        if (!span_ok(dB, (size_t)lddb * nrhs * CPLX)) return bad(h, dinfo, 6);
        if (!span_ok(dX, (size_t)lddx * nrhs * CPLX)) return bad(h, dinfo, 8);
        if (!span_ok(dWorkspace, need)) return bad(h, dinfo, 10);
        const CqRegion regions[2] = {{dA, m, n, ldda, 0, 4}, {dB, m, nrhs, lddb, 0, 6}};
        aclsolverStatus_t st = screen(h, dinfo, regions, 2);
        if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        return finish(launch_cgels(m, n, nrhs, reinterpret_cast<float2 *>(dA), ldda,
                                   reinterpret_cast<const float2 *>(dB), lddb, reinterpret_cast<float2 *>(dX), lddx,
                                   static_cast<float2 *>(dWorkspace), dinfo, h->stream));
    }
}
