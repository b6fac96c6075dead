/* solver_adapter.h -- the test-harness adapter protocol, version 2, as the reference's tests
 * define it (test/sgetrf/solver_adapter.h:25-69 of the reference; the same header is copied
 * beside each of its adapters).  An adapter is a shared library for ONE operation that an
 * external harness loads to drive the operation's public entry point: the harness owns the
 * aclsolver handle and its stream, hands the adapter compact row-major HOST buffers, and the
 * adapter marshals them to the operation's own device layout, runs the entry point once per
 * execute call, and reads the outputs back.
 *
 * The structures and functions must match the reference's field for field (the harness is
 * compiled against that header); this file restates them for this build.  The adapters of
 * this build (ops-solver_b200/adapter/real_lu_adapter.cpp) implement sgetrf, sgetri,
 * sgetribatched and smatinvbatched.
 *
 * Adapter return codes: 0 success, 1 invalid case, 2 allocation failed, 3 runtime (copy or
 * synchronisation) failed, 4 workspace query failed -- separate from the entry point's own
 * status, which execute returns through dut_status unchanged. */
#ifndef SOLVER_ADAPTER_H
#define SOLVER_ADAPTER_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C"
{
#endif
#define SOLVER_ADAPTER_VERSION 1u
#define SOLVER_ADAPTER_VERSION_V2 2u

    /* What the adapter drives: operation name, element type, where the operation's buffers
     * live and how they are laid out, whether info is one value or one per matrix, and the
     * address of the public function it calls. */
    typedef struct
    {
        uint32_t version, struct_size;
        const char *op, *dtype, *dut_abi, *dut_layout, *info_kind;
        const void *target_symbol;
    } SolverAdapterDesc;

    /* One test case (version 1 fields). */
    typedef struct
    {
        uint32_t version, struct_size;
        int64_t n, nrhs, batch, lda, ldb;
        char uplo;
        const char *info_probe, *input_kind;
        size_t a_bytes, b_bytes, out_bytes, info_count;
    } SolverAdapterCase;

    /* Version 2 case: the version 1 fields, then the extra shape, side / transpose and the
     * pivot and tau counts (pivots int32, 1-based; zero counts select the null-pivot path). */
    typedef struct
    {
        SolverAdapterCase base;
        int64_t m, k, ldc, ldx;
        char side, trans;
        size_t in_ipiv_count, in_tau_count, out_ipiv_count, out_tau_count;
    } SolverAdapterCaseV2;

    const SolverAdapterDesc *solver_adapter_descriptor(void);
    /* Allocates the case's device buffers; publishes the state before anything can fail, so
     * that solver_adapter_destroy can release a partly built one. */
    int solver_adapter_create_v2(const SolverAdapterCaseV2 *c, void *handle, void *stream, void **state);
    /* Restores every input, output, info and pivot buffer from the host transport; never
     * calls the operation. */
    int solver_adapter_reset_v2(void *state, const void *a, size_t a_bytes, const void *b, size_t b_bytes,
                                const int32_t *ipiv, size_t ipiv_count, const void *tau, size_t tau_bytes);
    /* Calls the operation once; its status is returned unchanged through dut_status. */
    int solver_adapter_execute(void *state, int *dut_status);
    /* After the harness has synchronised the stream: outputs, info and pivots to the host. */
    int solver_adapter_readback_v2(void *state, void *out, size_t out_bytes, int32_t *info, size_t info_count,
                                   int32_t *ipiv, size_t ipiv_count, void *tau, size_t tau_bytes);
    /* Releases the state (NULL or partly built is valid). */
    int solver_adapter_destroy(void *state);
#ifdef __cplusplus
}
#endif
#endif
