// api_qr.cpp -- real QR family C entry points: Sgeqrf, Sorgqr, Sormqr (+ _bufferSize) and
// SSgels (+ _bufferSize).
//
// Argument ladders follow the reference host code (paths relative to the reference root):
//   Sgeqrf    src/sgeqrf/arch35/sgeqrf_host.cpp:66-257 (CheckShape, m <= 8192 else NOT_SUPPORTED)
//   Sorgqr    src/sorgqr/arch35/sorgqr_host.cpp:88-252 (m <= 4096, 0 <= k <= n <= m)
//   Sormqr    src/sormqr/arch35/sormqr_host.cpp:100-316 (nq <= 4096, k <= nq)
//   SSgels    src/sgels/arch35/sgels_host.cpp:110-352 (m >= n, m, n <= 4096, nrhs <= 128,
//             niter set to 0, dX may overlap neither dB nor dA)
//   Xlarft    src/xlarft/arch35/xlarft_host.cpp:84-247 (params NULL, COLUMNWISE, FP32 only,
//             n <= 4096, k <= 256, no devInfo)
// An argument error writes -i (i counted without the handle) to the info buffer when that
// buffer is usable and returns INVALID_VALUE; shapes over the kernel limits return
// NOT_SUPPORTED (SSgels: INVALID_VALUE with -1 / -3, as the reference).  Workspace sizes are
// this build's: one 32 x 32 block factor (two for Sgeqrf and SSgels, whose look-ahead keeps
// consecutive panels' factors), plus the reflector copy (Sorgqr) or tau and Q^T B (SSgels).
#include <stdio.h>

#include <algorithm>

#include "handle.h"
#include "launch.h"
#include "launch_qr.h"

using namespace ops_solver;

namespace
{
constexpr int GEQRF_MAX_ROWS = 8192;
constexpr int Q_MAX = 4096;
constexpr int GELS_MAX_DIM = 4096;
constexpr int GELS_MAX_RHS = 128;

bool span_ok(const void *p, size_t bytes, size_t align)
{
    return p && reinterpret_cast<uintptr_t>(p) % align == 0 && is_device_pointer(p) && device_span(p, bytes);
}

bool overlap(const void *a, size_t abytes, const void *b, size_t bbytes)
{
    uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    return x <= y ? y - x < abytes : x - y < bbytes;
}

// -argument into a usable info buffer; `status` returned.
aclsolverStatus_t bad(Handle *h, int *info, int argument, aclsolverStatus_t status = ACLSOLVER_STATUS_INVALID_VALUE)
{
    if (span_ok(info, sizeof(int), alignof(int)) && launch_fill_info(info, -argument, 1, h->stream) != cudaSuccess)
        cudaGetLastError();
    return status;
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

int geqrf_shape(int m, int n, int lda)
{
    if (m < 0) return 1;
    if (n < 0) return 2;
    if (lda < std::max(1, m)) return 4;
    return 0;
}

int orgqr_shape(int m, int n, int k, int lda)
{
    if (m < 0) return 1;
    if (n < 0 || n > m) return 2;
    if (k < 0 || k > n) return 3;
    if (lda < std::max(1, m)) return 5;
    return 0;
}

int ormqr_shape(int side, int trans, int m, int n, int k, int lda, int ldc)
{
    if (side != ACLSOLVER_SIDE_LEFT && side != ACLSOLVER_SIDE_RIGHT) return 1;
    if (trans != ACLSOLVER_OP_N && trans != ACLSOLVER_OP_T && trans != ACLSOLVER_OP_C) return 2;
    if (m < 0) return 3;
    if (n < 0) return 4;
    const int nq = side == ACLSOLVER_SIDE_LEFT ? m : n;
    if (k < 0 || k > nq) return 5;
    if (lda < std::max(1, nq)) return 7;
    if (ldc < std::max(1, m)) return 10;
    return 0;
}

constexpr int64_t XLARFT_MAX_N = 4096;
constexpr int64_t XLARFT_MAX_K = 256;

aclsolverStatus_t xlarft_args(aclsolverParams_t params, int direct, int storev, int64_t n, int64_t k, int64_t ldv,
                              int64_t ldt, int dv, int dtau, int dt, int dc)
{
    if (params != nullptr) return ACLSOLVER_STATUS_INVALID_VALUE;
    if (direct != ACLSOLVER_DIRECT_FORWARD && direct != ACLSOLVER_DIRECT_BACKWARD) return ACLSOLVER_STATUS_INVALID_VALUE;
    if (storev != ACLSOLVER_STOREV_COLUMNWISE) return ACLSOLVER_STATUS_INVALID_VALUE;
    if (n < 0 || k < 0 || n < k) return ACLSOLVER_STATUS_INVALID_VALUE;
    if (ldv < std::max<int64_t>(1, n) || ldt < std::max<int64_t>(1, k)) return ACLSOLVER_STATUS_INVALID_VALUE;
    if (ldv > INT32_MAX || ldt > INT32_MAX) return ACLSOLVER_STATUS_INVALID_VALUE;
    if (dv != ACLSOLVER_R_32F || dtau != ACLSOLVER_R_32F || dt != ACLSOLVER_R_32F || dc != ACLSOLVER_R_32F)
        return ACLSOLVER_STATUS_NOT_SUPPORTED;
    return ACLSOLVER_STATUS_SUCCESS;
}

int gels_shape(int m, int n, int nrhs, int lda, int ldb, int ldx)
{
    if (m < 0 || m < n) return 1;
    if (n < 0) return 2;
    if (nrhs < 0) return 3;
    if (lda < std::max(1, m)) return 5;
    if (ldb < std::max(1, m)) return 7;
    if (ldx < std::max(1, n)) return 9;
    return 0;
}
}  // namespace

extern "C"
{
    aclsolverStatus_t aclsolverSgeqrf_bufferSize(aclsolverHandle_t handle, int m, int n, float *A, int lda, int *Lwork)
    {
        (void)handle;
        (void)A;
        if (!Lwork || geqrf_shape(m, n, lda)) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (m == 0 || n == 0)
        {
            *Lwork = 0;
            return ACLSOLVER_STATUS_SUCCESS;
        }
        if (m > GEQRF_MAX_ROWS) return ACLSOLVER_STATUS_NOT_SUPPORTED;
        *Lwork = QR_GEQRF_T_FLOATS;
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverSgeqrf(aclsolverHandle_t handle, int m, int n, float *A, int lda, float *TAU,
                                      float *Workspace, int Lwork, int *devInfo)
    {
        if (!devInfo) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        if (int b = geqrf_shape(m, n, lda)) return bad(h, devInfo, b);
        if (m == 0 || n == 0) return info_zero(h, devInfo);
        if (!A) return bad(h, devInfo, 3);
        if (!TAU) return bad(h, devInfo, 5);
        if (m > GEQRF_MAX_ROWS) return bad(h, devInfo, 1, ACLSOLVER_STATUS_NOT_SUPPORTED);
        if (!Workspace) return bad(h, devInfo, 6);
        if (Lwork < QR_GEQRF_T_FLOATS) return bad(h, devInfo, 7);
        if (!span_ok(A, (size_t)lda * n * sizeof(float), alignof(float))) return bad(h, devInfo, 3);
        if (!span_ok(TAU, (size_t)std::min(m, n) * sizeof(float), alignof(float))) return bad(h, devInfo, 5);
        if (!span_ok(Workspace, (size_t)QR_GEQRF_T_FLOATS * sizeof(float), alignof(float)))
            return bad(h, devInfo, 6);
        if (!span_ok(devInfo, sizeof(int), alignof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
        aclsolverStatus_t st = info_zero(h, devInfo);
        if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        return finish(launch_sgeqrf(A, lda, m, n, TAU, Workspace, h->stream));
    }

    aclsolverStatus_t aclsolverSorgqr_bufferSize(aclsolverHandle_t handle, int m, int n, int k, const float *A,
                                                 int lda, const float *tau, int *lwork)
    {
        (void)handle;
        (void)A;
        (void)tau;
        if (!lwork || orgqr_shape(m, n, k, lda)) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (m == 0 || n == 0)
        {
            *lwork = 0;
            return ACLSOLVER_STATUS_SUCCESS;
        }
        if (m > Q_MAX) return ACLSOLVER_STATUS_NOT_SUPPORTED;
        *lwork = m * k + QR_T_FLOATS;
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverSorgqr(aclsolverHandle_t handle, int m, int n, int k, float *A, int lda,
                                      const float *tau, float *work, int lwork, int *devInfo)
    {
        if (!devInfo) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        if (int b = orgqr_shape(m, n, k, lda)) return bad(h, devInfo, b);
        if (m == 0 || n == 0) return info_zero(h, devInfo);
        if (!A) return bad(h, devInfo, 4);
        if (k > 0 && !tau) return bad(h, devInfo, 6);
        if (m > Q_MAX) return bad(h, devInfo, 1, ACLSOLVER_STATUS_NOT_SUPPORTED);
        const size_t need = (size_t)m * k + QR_T_FLOATS;
        if (!work) return bad(h, devInfo, 7);
        if ((size_t)std::max(lwork, 0) < need) return bad(h, devInfo, 8);
        if (!span_ok(A, (size_t)lda * n * sizeof(float), alignof(float))) return bad(h, devInfo, 4);
        if (k > 0 && !span_ok(tau, (size_t)k * sizeof(float), alignof(float))) return bad(h, devInfo, 6);
        if (!span_ok(work, need * sizeof(float), alignof(float))) return bad(h, devInfo, 7);
        if (!span_ok(devInfo, sizeof(int), alignof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
        aclsolverStatus_t st = info_zero(h, devInfo);
        if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        return finish(launch_sorgqr(m, n, k, A, lda, tau, work, h->stream));
    }

    aclsolverStatus_t aclsolverSormqr_bufferSize(aclsolverHandle_t handle, aclsolverSideMode_t side,
                                                 aclsolverOperation_t trans, int m, int n, int k, const float *A,
                                                 int lda, const float *tau, const float *C, int ldc, int *lwork)
    {
        (void)handle;
        (void)A;
        (void)tau;
        (void)C;
        if (!lwork || ormqr_shape(side, trans, m, n, k, lda, ldc)) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (m == 0 || n == 0 || k == 0)
        {
            *lwork = 0;
            return ACLSOLVER_STATUS_SUCCESS;
        }
        if ((side == ACLSOLVER_SIDE_LEFT ? m : n) > Q_MAX) return ACLSOLVER_STATUS_NOT_SUPPORTED;
        *lwork = QR_T_FLOATS;
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverSormqr(aclsolverHandle_t handle, aclsolverSideMode_t side, aclsolverOperation_t trans,
                                      int m, int n, int k, const float *A, int lda, const float *tau, float *C,
                                      int ldc, float *work, int lwork, int *devInfo)
    {
        if (!devInfo) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        if (int b = ormqr_shape(side, trans, m, n, k, lda, ldc)) return bad(h, devInfo, b);
        if (m == 0 || n == 0 || k == 0) return info_zero(h, devInfo);
        if (!A) return bad(h, devInfo, 6);
        if (!tau) return bad(h, devInfo, 8);
        if (!C) return bad(h, devInfo, 9);
        const int nq = side == ACLSOLVER_SIDE_LEFT ? m : n;
        if (nq > Q_MAX) return bad(h, devInfo, 5, ACLSOLVER_STATUS_NOT_SUPPORTED);
        if (!work) return bad(h, devInfo, 11);
        if (lwork < QR_T_FLOATS) return bad(h, devInfo, 12);
        if (!span_ok(A, (size_t)lda * k * sizeof(float), alignof(float))) return bad(h, devInfo, 6);
        if (!span_ok(tau, (size_t)k * sizeof(float), alignof(float))) return bad(h, devInfo, 8);
        if (!span_ok(C, (size_t)ldc * n * sizeof(float), alignof(float))) return bad(h, devInfo, 9);
        if (!span_ok(work, (size_t)QR_T_FLOATS * sizeof(float), alignof(float))) return bad(h, devInfo, 11);
        if (!span_ok(devInfo, sizeof(int), alignof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
        aclsolverStatus_t st = info_zero(h, devInfo);
        if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        return finish(launch_sormqr(side == ACLSOLVER_SIDE_RIGHT, trans != ACLSOLVER_OP_N, m, n, k, A, lda, tau, C,
                                    ldc, work, h->stream));
    }

    aclsolverStatus_t aclsolverXlarft_bufferSize(aclsolverHandle_t handle, aclsolverParams_t params,
                                                 aclsolverDirectMode_t direct, aclsolverStorevMode_t storev, int64_t n,
                                                 int64_t k, aclsolverDataType_t dataTypeV, const void *V, int64_t ldv,
                                                 aclsolverDataType_t dataTypeTau, const void *tau,
                                                 aclsolverDataType_t dataTypeT, void *T, int64_t ldt,
                                                 aclsolverDataType_t computeType, size_t *workspaceInBytesOnDevice,
                                                 size_t *workspaceInBytesOnHost)
    {
        (void)handle;
        (void)V;
        (void)tau;
        (void)T;
        if (!workspaceInBytesOnDevice || !workspaceInBytesOnHost) return ACLSOLVER_STATUS_INVALID_VALUE;
        aclsolverStatus_t st = xlarft_args(params, direct, storev, n, k, ldv, ldt, dataTypeV, dataTypeTau, dataTypeT,
                                           computeType);
        if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        *workspaceInBytesOnHost = 0;
        if (n == 0 || k == 0)
        {
            *workspaceInBytesOnDevice = 0;
            return ACLSOLVER_STATUS_SUCCESS;
        }
        if (n > XLARFT_MAX_N || k > XLARFT_MAX_K) return ACLSOLVER_STATUS_NOT_SUPPORTED;
        *workspaceInBytesOnDevice = xlarft_work_bytes((int)k);
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverXlarft(aclsolverHandle_t handle, aclsolverParams_t params, aclsolverDirectMode_t direct,
                                      aclsolverStorevMode_t storev, int64_t n, int64_t k, aclsolverDataType_t dataTypeV,
                                      const void *V, int64_t ldv, aclsolverDataType_t dataTypeTau, const void *tau,
                                      aclsolverDataType_t dataTypeT, void *T, int64_t ldt,
                                      aclsolverDataType_t computeType, void *bufferOnDevice,
                                      size_t workspaceInBytesOnDevice, void *bufferOnHost,
                                      size_t workspaceInBytesOnHost)
    {
        (void)bufferOnHost;
        (void)workspaceInBytesOnHost;
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        aclsolverStatus_t st = xlarft_args(params, direct, storev, n, k, ldv, ldt, dataTypeV, dataTypeTau, dataTypeT,
                                           computeType);
        if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        if (n == 0 || k == 0) return ACLSOLVER_STATUS_SUCCESS;
        if (n > XLARFT_MAX_N || k > XLARFT_MAX_K) return ACLSOLVER_STATUS_NOT_SUPPORTED;
        if (!V || !tau || !T || !bufferOnDevice) return ACLSOLVER_STATUS_INVALID_VALUE;
        const size_t need = xlarft_work_bytes((int)k);
        if (workspaceInBytesOnDevice < need) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (!span_ok(V, (size_t)ldv * k * sizeof(float), alignof(float)) ||
            !span_ok(tau, (size_t)k * sizeof(float), alignof(float)) ||
            !span_ok(T, (size_t)ldt * k * sizeof(float), alignof(float)) ||
            !span_ok(bufferOnDevice, need, alignof(float)))
            return ACLSOLVER_STATUS_INVALID_VALUE;
        return finish(launch_xlarft(direct == ACLSOLVER_DIRECT_BACKWARD, (int)n, (int)k, static_cast<const float *>(V),
                                    (int)ldv, static_cast<const float *>(tau), static_cast<float *>(T), (int)ldt,
                                    static_cast<float *>(bufferOnDevice), h->stream));
    }

    aclsolverStatus_t aclsolverSSgels_bufferSize(aclsolverHandle_t handle, int m, int n, int nrhs, float *dA, int ldda,
                                                 float *dB, int lddb, float *dX, int lddx, void *dwork,
                                                 size_t *lwork_bytes)
    {
        (void)dA;
        (void)dB;
        (void)dX;
        (void)dwork;
        if (!lwork_bytes) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        if (gels_shape(m, n, nrhs, ldda, lddb, lddx)) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (m == 0 || n == 0 || nrhs == 0)
        {
            *lwork_bytes = 0;
            return ACLSOLVER_STATUS_SUCCESS;
        }
        if (m > GELS_MAX_DIM || n > GELS_MAX_DIM || nrhs > GELS_MAX_RHS) return ACLSOLVER_STATUS_INVALID_VALUE;
        *lwork_bytes = sgels_work_floats(m, n, nrhs) * sizeof(float);
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverSSgels(aclsolverHandle_t handle, int m, int n, int nrhs, float *dA, int ldda, float *dB,
                                      int lddb, float *dX, int lddx, void *dWorkspace, size_t lwork_bytes, int *niter,
                                      int *dinfo)
    {
        if (!dinfo) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        if (!niter) return bad(h, dinfo, 12);
        *niter = 0;  // a direct QR solve: no refinement iterations
        if (int b = gels_shape(m, n, nrhs, ldda, lddb, lddx)) return bad(h, dinfo, b);
        if (m == 0 || n == 0 || nrhs == 0) return info_zero(h, dinfo);
        if (!dA) return bad(h, dinfo, 4);
        if (!dB) return bad(h, dinfo, 6);
        if (!dX) return bad(h, dinfo, 8);
        const size_t xb = (size_t)nrhs * lddx * sizeof(float);
        if (overlap(dX, xb, dB, (size_t)nrhs * lddb * sizeof(float)) ||
            overlap(dX, xb, dA, (size_t)n * ldda * sizeof(float)))
            return bad(h, dinfo, 8);
        if (m > GELS_MAX_DIM || n > GELS_MAX_DIM) return bad(h, dinfo, 1);
        if (nrhs > GELS_MAX_RHS) return bad(h, dinfo, 3);
        const size_t need = sgels_work_floats(m, n, nrhs) * sizeof(float);
        if (!dWorkspace) return bad(h, dinfo, 10);
        if (lwork_bytes < need) return bad(h, dinfo, 11);
        if (!span_ok(dA, (size_t)ldda * n * sizeof(float), alignof(float))) return bad(h, dinfo, 4);
        if (!span_ok(dB, (size_t)lddb * nrhs * sizeof(float), alignof(float))) return bad(h, dinfo, 6);
        if (!span_ok(dX, xb, alignof(float))) return bad(h, dinfo, 8);
        if (!span_ok(dWorkspace, need, alignof(float))) return bad(h, dinfo, 10);
        if (!span_ok(dinfo, sizeof(int), alignof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
        aclsolverStatus_t st = info_zero(h, dinfo);
        if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        return finish(launch_sgels(m, n, nrhs, dA, ldda, dB, lddb, dX, lddx, static_cast<float *>(dWorkspace),
                                   h->stream));
    }
}
