// real_lu_adapter.cpp -- the harness adapter protocol (include/solver_adapter.h; reference
// test/sgetrf/solver_adapter.h) for this library's real LU entries, so that an external
// harness written for the reference's adapters (test/sgetrf/sgetrf_adapter.cpp and its
// sgetri, sgetri_batched and smatinv_batched siblings) drives this build unchanged.  Built
// once per operation with ADAPTER_OP = 0 (aclsolverSgetrf), 1 (aclsolverSgetri),
// 2 (aclsolverSgetriBatched) or 3 (aclsolverSmatinvBatched) into
// lib/libsolver_adapter_<op>.so.
//
// Transport: compact row-major host matrices (m x n each, batch of them back to back), int32
// 1-based pivots, int32 info.  Device side, as the operation takes them: column-major with
// leading dimension lda (ldc for the batched outputs), the rows past m of each column filled
// with a padding sentinel so that a write outside the matrix shows in the readback; batched
// operations get device pointer tables; outputs, info and pivots start as a 0xA5 byte pattern
// so that an unwritten entry shows too.  All copies run on the harness's stream (it must be
// the handle's stream), and reset waits for them, so the operation sees its inputs in place.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <new>
#include <vector>

#include "cann_ops_solver.h"
#include "solver_adapter.h"

#ifndef ADAPTER_OP
#error "ADAPTER_OP selects the operation: 0 sgetrf, 1 sgetri, 2 sgetri_batched, 3 smatinv_batched"
#endif

namespace
{
enum Op
{
    SGETRF = 0,
    SGETRI = 1,
    SGETRI_BATCHED = 2,
    SMATINV_BATCHED = 3
};
constexpr Op OP = static_cast<Op>(ADAPTER_OP);
constexpr bool BATCHED = OP == SGETRI_BATCHED || OP == SMATINV_BATCHED;
constexpr bool FACTOR = OP == SGETRF;
constexpr bool LU_INPUT = OP == SGETRI || OP == SGETRI_BATCHED;  // the input is a factor (+ pivots)
constexpr bool IN_PLACE = !BATCHED;
constexpr float PAD = -773.0f;  // the padding value the reference's harness uses
constexpr int FILL = 0xA5;      // unwritten-output byte pattern

enum Result
{
    OK = 0,
    INVALID_CASE = 1,
    ALLOC_FAILED = 2,
    RUNTIME_FAILED = 3,
    QUERY_FAILED = 4
};

struct Buffer
{
    void *p = nullptr;
    size_t bytes = 0;
    bool alloc(size_t n)
    {
        bytes = n;
        return n == 0 || cudaMalloc(&p, n) == cudaSuccess;
    }
    bool release()
    {
        if (p && cudaFree(p) != cudaSuccess) return false;
        p = nullptr;
        bytes = 0;
        return true;
    }
};

struct State
{
    aclsolverHandle_t handle = nullptr;
    cudaStream_t stream = nullptr;
    int m = 0, n = 0, lda = 0, ldc = 0, batch = 0, lwork = 0;
    size_t cells = 0;                   // transport elements per matrix (m n)
    size_t a_stride = 0, c_stride = 0;  // device elements per matrix (lda n, ldc n)
    size_t transport_bytes = 0, info_count = 0, in_piv = 0, out_piv = 0;
    bool ready = false, reset = false, pending = false;
    Buffer a, c, work, piv, info, a_tab, c_tab;
    std::vector<float> host;  // column-major staging of every matrix of the case
};

bool mul(size_t x, size_t y, size_t &out)
{
    if (y != 0 && x > SIZE_MAX / y) return false;
    out = x * y;
    return true;
}
bool fits_int(int64_t v) { return v >= 0 && v <= INT_MAX; }

// The case against this build's limits for the operation (those of its public entry).
bool validate(const SolverAdapterCaseV2 *c, State &s)
{
    if (!c || c->base.version != SOLVER_ADAPTER_VERSION_V2 || c->base.struct_size != sizeof(*c)) return false;
    if (!fits_int(c->base.n) || !fits_int(c->base.batch) || !fits_int(c->base.lda)) return false;
    if (c->base.b_bytes != 0 || c->in_tau_count != 0 || c->out_tau_count != 0) return false;
    if (!BATCHED && c->base.batch != 1) return false;
    s.n = (int)c->base.n;
    s.batch = (int)c->base.batch;
    s.lda = (int)c->base.lda;
    if (FACTOR)
    {
        if (!fits_int(c->m) || c->m > 8192) return false;
        s.m = (int)c->m;
    }
    else
    {
        if ((c->m != 0 && c->m != s.n) || s.n > (OP == SMATINV_BATCHED ? 32 : 4096)) return false;
        s.m = s.n;
    }
    if (s.lda < std::max(1, s.m)) return false;
    s.ldc = s.lda;
    if (BATCHED)
    {
        if (!fits_int(c->ldc) || c->ldc < std::max(1, s.n)) return false;
        s.ldc = (int)c->ldc;
    }
    size_t total = 0, pivots = 0;
    if (!mul((size_t)s.m, (size_t)s.n, s.cells) || !mul(s.cells, (size_t)s.batch, total) ||
        !mul(total, sizeof(float), s.transport_bytes) ||
        !mul((size_t)std::min(s.m, s.n), (size_t)s.batch, pivots) || !mul((size_t)s.lda, (size_t)s.n, s.a_stride) ||
        !mul((size_t)s.ldc, (size_t)s.n, s.c_stride))
        return false;
    s.info_count = BATCHED ? (size_t)s.batch : 1;
    if (c->base.info_count != s.info_count || c->base.a_bytes != s.transport_bytes ||
        c->base.out_bytes != s.transport_bytes)
        return false;
    // pivots: produced by the factorisation, consumed by sgetri / sgetri_batched, none for
    // smatinv; a zero count selects the entry's null-pivot path
    if (FACTOR && !(c->in_ipiv_count == 0 && (c->out_ipiv_count == 0 || c->out_ipiv_count == pivots))) return false;
    if (LU_INPUT && !(c->out_ipiv_count == 0 && (c->in_ipiv_count == 0 || c->in_ipiv_count == pivots))) return false;
    if (OP == SMATINV_BATCHED && (c->in_ipiv_count != 0 || c->out_ipiv_count != 0)) return false;
    s.in_piv = c->in_ipiv_count;
    s.out_piv = c->out_ipiv_count;
    return true;
}

aclsolverStatus_t query_workspace(State &s)
{
    s.lwork = 0;
    if (FACTOR) return aclsolverSgetrf_bufferSize(s.handle, s.m, s.n, nullptr, s.lda, &s.lwork);
    if (OP == SGETRI) return aclsolverSgetri_bufferSize(s.handle, s.n, nullptr, s.lda, &s.lwork);
    return ACLSOLVER_STATUS_SUCCESS;
}

int allocate(State &s)
{
    if (query_workspace(s) != ACLSOLVER_STATUS_SUCCESS || s.lwork < 0) return QUERY_FAILED;
    size_t a_bytes = 0, c_bytes = 0, host_cells = 0;
    if (!mul(s.a_stride, (size_t)s.batch, host_cells) || !mul(host_cells, sizeof(float), a_bytes)) return ALLOC_FAILED;
    if (!IN_PLACE && !mul(s.c_stride * sizeof(float), (size_t)s.batch, c_bytes)) return ALLOC_FAILED;
    const size_t tables = BATCHED ? (size_t)s.batch * sizeof(void *) : 0;
    if (!s.a.alloc(a_bytes) || !s.c.alloc(c_bytes) || !s.work.alloc((size_t)s.lwork * sizeof(float)) ||
        !s.piv.alloc(std::max(s.in_piv, s.out_piv) * sizeof(int32_t)) || !s.info.alloc(s.info_count * sizeof(int32_t)) ||
        !s.a_tab.alloc(tables) || !s.c_tab.alloc(tables))
        return ALLOC_FAILED;
    s.host.resize(std::max(host_cells, !IN_PLACE ? s.c_stride * (size_t)s.batch : 0));
    s.ready = true;
    return OK;
}

bool sync(State &s)
{
    if (cudaStreamSynchronize(s.stream) != cudaSuccess) return false;
    s.pending = false;
    return true;
}

bool upload_tables(State &s)
{
    if (!BATCHED || s.batch == 0) return true;
    std::vector<const void *> at((size_t)s.batch), ct((size_t)s.batch);
    for (int q = 0; q < s.batch; ++q)
    {
        at[q] = static_cast<const float *>(s.a.p) + (size_t)q * s.a_stride;
        ct[q] = static_cast<const float *>(s.c.p) + (size_t)q * s.c_stride;
    }
    return cudaMemcpyAsync(s.a_tab.p, at.data(), s.a_tab.bytes, cudaMemcpyHostToDevice, s.stream) == cudaSuccess &&
           cudaMemcpyAsync(s.c_tab.p, ct.data(), s.c_tab.bytes, cudaMemcpyHostToDevice, s.stream) == cudaSuccess &&
           sync(s);  // the host tables must outlive the copies
}

bool upload(State &s, const float *rows, const int32_t *ipiv, size_t ipiv_count)
{
    // row-major transport -> column-major device image, padding rows past m with PAD
    std::fill(s.host.begin(), s.host.begin() + (ptrdiff_t)(s.a_stride * (size_t)s.batch), PAD);
    for (int q = 0; q < s.batch; ++q)
    {
        const float *src = rows + (size_t)q * s.cells;
        float *dst = s.host.data() + (size_t)q * s.a_stride;
        for (int i = 0; i < s.m; ++i)
            for (int j = 0; j < s.n; ++j) dst[(size_t)j * s.lda + i] = src[(size_t)i * s.n + j];
    }
    bool ok = s.a.bytes == 0 ||
              cudaMemcpyAsync(s.a.p, s.host.data(), s.a.bytes, cudaMemcpyHostToDevice, s.stream) == cudaSuccess;
    ok = ok && (s.c.bytes == 0 || cudaMemsetAsync(s.c.p, FILL, s.c.bytes, s.stream) == cudaSuccess);
    ok = ok && (s.work.bytes == 0 || cudaMemsetAsync(s.work.p, 0, s.work.bytes, s.stream) == cudaSuccess);
    ok = ok && (s.info.bytes == 0 || cudaMemsetAsync(s.info.p, FILL, s.info.bytes, s.stream) == cudaSuccess);
    ok = ok && (s.piv.bytes == 0 || cudaMemsetAsync(s.piv.p, FILL, s.piv.bytes, s.stream) == cudaSuccess);
    ok = ok && (ipiv_count == 0 || cudaMemcpyAsync(s.piv.p, ipiv, ipiv_count * sizeof(int32_t),
                                                   cudaMemcpyHostToDevice, s.stream) == cudaSuccess);
    return ok && sync(s) && upload_tables(s);
}

bool download(State &s, float *rows)
{
    const Buffer &src = IN_PLACE ? s.a : s.c;
    const size_t stride = IN_PLACE ? s.a_stride : s.c_stride;
    const int ld = IN_PLACE ? s.lda : s.ldc;
    if (src.bytes == 0) return true;
    if (cudaMemcpyAsync(s.host.data(), src.p, src.bytes, cudaMemcpyDeviceToHost, s.stream) != cudaSuccess || !sync(s))
        return false;
    for (int q = 0; q < s.batch; ++q)
    {
        const float *col = s.host.data() + (size_t)q * stride;
        float *dst = rows + (size_t)q * s.cells;
        for (int i = 0; i < s.m; ++i)
            for (int j = 0; j < s.n; ++j) dst[(size_t)i * s.n + j] = col[(size_t)j * ld + i];
    }
    return true;
}

bool download_ints(State &s, const Buffer &b, int32_t *out, size_t count)
{
    if (count == 0) return true;
    return cudaMemcpyAsync(out, b.p, count * sizeof(int32_t), cudaMemcpyDeviceToHost, s.stream) == cudaSuccess &&
           sync(s);
}

aclsolverStatus_t run(State &s)
{
    float *a = static_cast<float *>(s.a.p);
    int *piv = s.piv.bytes ? static_cast<int *>(s.piv.p) : nullptr;
    int *info = static_cast<int *>(s.info.p);
    if constexpr (OP == SGETRF)
        return aclsolverSgetrf(s.handle, s.m, s.n, a, s.lda, static_cast<float *>(s.work.p),
                               s.out_piv ? piv : nullptr, info);
    else if constexpr (OP == SGETRI)
        return aclsolverSgetri(s.handle, s.n, a, s.lda, s.in_piv ? piv : nullptr, static_cast<float *>(s.work.p),
                               s.lwork, info);
    else if constexpr (OP == SGETRI_BATCHED)
        return aclsolverSgetriBatched(s.handle, s.n, static_cast<const float *const *>(s.a_tab.p), s.lda,
                                      s.in_piv ? piv : nullptr, static_cast<float *const *>(s.c_tab.p), s.ldc, info,
                                      s.batch);
    else
        return aclsolverSmatinvBatched(s.handle, s.n, static_cast<const float *const *>(s.a_tab.p), s.lda,
                                       static_cast<float *const *>(s.c_tab.p), s.ldc, info, s.batch);
}

const void *target()
{
    if constexpr (OP == SGETRF)
        return reinterpret_cast<const void *>(&aclsolverSgetrf);
    else if constexpr (OP == SGETRI)
        return reinterpret_cast<const void *>(&aclsolverSgetri);
    else if constexpr (OP == SGETRI_BATCHED)
        return reinterpret_cast<const void *>(&aclsolverSgetriBatched);
    else
        return reinterpret_cast<const void *>(&aclsolverSmatinvBatched);
}
}  // namespace

extern "C"
{
    __attribute__((visibility("default"))) const SolverAdapterDesc *solver_adapter_descriptor(void)
    {
        static const char *const names[] = {"sgetrf", "sgetri", "sgetribatched", "smatinvbatched"};
        static const SolverAdapterDesc desc{SOLVER_ADAPTER_VERSION_V2, sizeof(SolverAdapterDesc), names[OP], "float32",
                                            "device", "column_major", BATCHED ? "array" : "scalar", target()};
        return &desc;
    }

    __attribute__((visibility("default"))) int solver_adapter_create_v2(const SolverAdapterCaseV2 *c, void *handle,
                                                                         void *stream, void **state)
    {
        if (!state) return INVALID_CASE;
        *state = nullptr;
        if (!handle) return INVALID_CASE;
        State *s = new (std::nothrow) State;
        if (!s) return ALLOC_FAILED;
        *state = s;  // published first: destroy releases a partly built state
        s->handle = static_cast<aclsolverHandle_t>(handle);
        s->stream = static_cast<cudaStream_t>(stream);
        if (!validate(c, *s)) return INVALID_CASE;
        aclrtStream bound = nullptr;
        if (aclsolverGetStream(s->handle, &bound) != ACLSOLVER_STATUS_SUCCESS ||
            bound != static_cast<aclrtStream>(s->stream))
            return INVALID_CASE;
        try
        {
            return allocate(*s);
        }
        catch (const std::exception &)
        {
            return ALLOC_FAILED;
        }
    }

    __attribute__((visibility("default"))) int solver_adapter_reset_v2(void *state, const void *a, size_t a_bytes,
                                                                        const void *, size_t b_bytes,
                                                                        const int32_t *ipiv, size_t ipiv_count,
                                                                        const void *, size_t tau_bytes)
    {
        State *s = static_cast<State *>(state);
        if (!s || !s->ready || a_bytes != s->transport_bytes || (a_bytes && !a) || b_bytes != 0 ||
            ipiv_count != s->in_piv || (ipiv_count && !ipiv) || tau_bytes != 0)
            return INVALID_CASE;
        s->reset = false;
        if (s->pending && !sync(*s)) return RUNTIME_FAILED;
        if (!upload(*s, static_cast<const float *>(a), ipiv, ipiv_count)) return RUNTIME_FAILED;
        s->reset = true;
        return OK;
    }

    __attribute__((visibility("default"))) int solver_adapter_execute(void *state, int *dut_status)
    {
        State *s = static_cast<State *>(state);
        if (!s || !s->ready || !s->reset || !dut_status) return INVALID_CASE;
        s->pending = true;  // the entry may enqueue work even when it returns an error
        *dut_status = (int)run(*s);
        return OK;
    }

    __attribute__((visibility("default"))) int solver_adapter_readback_v2(void *state, void *out, size_t out_bytes,
                                                                           int32_t *info, size_t info_count,
                                                                           int32_t *ipiv, size_t ipiv_count, void *,
                                                                           size_t tau_bytes)
    {
        State *s = static_cast<State *>(state);
        if (!s || !s->ready || !s->reset || out_bytes != s->transport_bytes || (out_bytes && !out) ||
            info_count != s->info_count || (info_count && !info) || ipiv_count != s->out_piv ||
            (ipiv_count && !ipiv) || tau_bytes != 0)
            return INVALID_CASE;
        if (!download(*s, static_cast<float *>(out)) || !download_ints(*s, s->info, info, info_count) ||
            !download_ints(*s, s->piv, ipiv, ipiv_count))
            return RUNTIME_FAILED;
        return OK;
    }

    __attribute__((visibility("default"))) int solver_adapter_destroy(void *state)
    {
        State *s = static_cast<State *>(state);
        if (!s) return OK;
        if (s->pending && !sync(*s)) return RUNTIME_FAILED;  // kept for a retry
        bool freed = true;
        for (Buffer *b : {&s->c_tab, &s->a_tab, &s->info, &s->piv, &s->work, &s->c, &s->a}) freed = b->release() && freed;
        if (!freed)
        {
            s->ready = false;
            return RUNTIME_FAILED;
        }
        delete s;
        return OK;
    }
}
