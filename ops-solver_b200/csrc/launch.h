// launch.h -- the internal launcher interface between the host C++ layer (argument
// ladders, dispatch, scratch) and the CUDA kernels.  Plain pointers and sizes only.
//
// Every launcher enqueues on `stream` and returns the cudaError_t of the launch
// (cudaGetLastError after the <<<>>>), never synchronising.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ops_solver
{

// A batch of column-major float matrices: either a device pointer table (`table`, slot
// first+q) or a single matrix (`single`).
struct RealBatch
{
    float *single;
    float *const *table;
    int n;
    int ld;
    int first;
    int count;
};

// ---- real Cholesky ---------------------------------------------------------------------
// Fills info[0..count) with value.
cudaError_t launch_fill_info(int *info, int value, int64_t count, cudaStream_t stream);
// SpotrsBatched slot scan: info[0] = -4 if any A slot is null, else -6 if any B slot is
// null, else 0 (cholesky_simt.cpp:28-48 contract).
// The inverse from a Cholesky factor (potri.cu): diagonal check into info[0] and the n x n
// identity into w (ld n); then, after the solve, the selected triangle of A from w's lower
// triangle when info[0] == 0.
cudaError_t launch_potri_prepare(const float *a, int lda, int n, float *w, int *info, cudaStream_t stream);
cudaError_t launch_potri_store(float *a, int lda, int upper, int n, const float *w, const int *info,
                               cudaStream_t stream);
cudaError_t launch_cpotri_prepare(const float2 *a, int lda, int n, float2 *w, int *info, cudaStream_t stream);
cudaError_t launch_cpotri_store(float2 *a, int lda, int upper, int n, const float2 *w, const int *info,
                                cudaStream_t stream);
// flags: two device words that are zero on entry (left zero on exit).
cudaError_t launch_solve_slot_check(int *info, float *const *a, float *const *b, int count, int *flags,
                                    cudaStream_t stream);
// In-place Cholesky of n <= 32 matrices, per-slot info (null slot -> -3).
cudaError_t launch_potrf_small(const RealBatch &a, int upper, int *info, cudaStream_t stream);
// In-place Cholesky of n > 32 matrices (FMA order, left-looking), per-slot info.
// Real Cholesky above order 32 (potrf_blocked.cu): a block per matrix with the packed
// triangle in shared memory up to POTRF_PACKED_MAX; above, one matrix over the whole GPU
// (scratch: potrf_large_scratch_bytes, a backup of the lower triangle).
constexpr int POTRF_PACKED_MAX = 256;
cudaError_t launch_potrf_packed(const RealBatch &a, int upper, int *info, cudaStream_t stream);
size_t potrf_large_scratch_bytes(int n);
cudaError_t launch_potrf_large(float *A, int lda, int upper, int n, int *info, void *scratch, cudaStream_t stream);
// Cholesky solve for n > 32: dot-accumulate order (dot_order = 1) or right-looking order.
cudaError_t launch_potrs_generic(const RealBatch &a, const RealBatch &b, int nrhs, int upper, int dot_order,
                                 const int *info, cudaStream_t stream);
// Cholesky solve for n <= 32 (SolveKernel order), any nrhs; skipped when info[0] != 0.
cudaError_t launch_potrs_small(const RealBatch &a, const RealBatch &b, int nrhs, int upper, const int *info,
                               cudaStream_t stream);

// ---- real LU ---------------------------------------------------------------------------
// Batched LU of m x n matrices (a.n columns) for m, n <= 64.  ipiv: min(m, n) per matrix
// (nullptr = no pivoting).  info: first zero pivot, -2 for a null slot.
cudaError_t launch_getrf_small(const RealBatch &a, int m, int *ipiv, int *info, cudaStream_t stream);
// Batched LU solve for n <= 64; trans 0/1; ipiv n per matrix or nullptr.
cudaError_t launch_getrs_small(const RealBatch &a, const int *ipiv, const RealBatch &b, int nrhs, int trans,
                               int *info, cudaStream_t stream);
// Batched out-of-place inverse from LU for n <= 64 (c may alias a: the factors are staged
// in shared memory before the inverse is written).
cudaError_t launch_getri_small(const RealBatch &a, const int *ipiv, const RealBatch &c, int *info,
                               cudaStream_t stream);

// Blocked LU for 64 < n <= 512 (square), one 256-thread block per matrix.  mode 0: plain
// FP32, bit-identical to the unblocked order; 1: BF16 tensor-core trailing update; 3: split
// BF16 (three products).  ipiv n per matrix or nullptr; info as launch_getrf_small.
// src (optional): factor a copy of src[q] (leading dimension src_ld) into a's slot q.
// perm (optional): n per matrix, the composed row permutation (P b = b[perm]).
// lists (optional, for the blocked solve's `lists`): the factorisation's row changes panel by
// panel, and the L columns of each 128-column block keep the row order they had when the
// block was finished (the interchanges of later blocks are not applied to them, so ipiv and
// the factors are not in LAPACK form).  Per matrix BLOCKED_PANELS entries of
// PANEL_LIST_SHORTS shorts: [count, position[64], source[64], pad]; panel p moves the row at
// 32p + source[i] to 32p + position[i] (all moves of the entry at once).
constexpr int BLOCKED_MAX_N = 512;
constexpr int BLOCKED_SOLVE_MAX_N = 8192;  // the blocked solve: x of one right-hand side in shared memory
constexpr int BLOCKED_PANELS = BLOCKED_MAX_N / 32;
constexpr int BLOCKED_OUTER_COLS = 128;  // columns of the blocks whose L keeps its row order
constexpr int PANEL_LIST_SHORTS = 132;
cudaError_t launch_getrf_blocked(const RealBatch &a, int *ipiv, int *info, int mode, cudaStream_t stream,
                                 const float *const *src = nullptr, int src_ld = 0, int *perm = nullptr,
                                 short *lists = nullptr);
// Blocked LU solve (trans 0) for 64 < n <= 8192.  Row interchanges from ipiv (LAPACK form,
// applied in order) or, when perm is given, from the permutation perm (P b = b[perm], see
// launch_permutation); both may be null.  `skip` (nullptr = none): per (matrix,
// right-hand side) states; a group of right-hand sides whose states are all nonzero is
// skipped (iterative refinement).  info may be null.  lists (with ipiv and perm null):
// factors from launch_getrf_blocked with `lists`; the forward sweep applies each 128-column
// block's row changes to the vectors before that block's columns.
// ---- large single-matrix LU (lu_large.cu) ---------------------------------------------
constexpr int LARGE_MAX_ROWS = 8192;  // up to four panel rows per thread of an 8 x 256-thread cluster
constexpr int LARGE_MAX_COLS = 8192;
constexpr int LARGE_WAIT_ERROR = -1000;  // info when a cluster panel's bounded wait ran out
// Device scratch of one factorisation: info, per 32-column panel its zero-pivot bits and
// its changed positions (position, physical row), at most 64.
struct LargeStatus
{
    int info;
    int error;  // a bounded wait of the cluster panel ran out (the factors are not valid)
    int pad[2];
    unsigned zmask[LARGE_MAX_COLS / 32];
    int nchg[LARGE_MAX_COLS / 32];
    int2 chg[LARGE_MAX_COLS / 32][64];
};
// P A = L U of one m x n matrix (n <= m <= LARGE_MAX_ROWS) over the whole GPU; ipiv may be
// null (no pivoting); *info receives the first zero pivot (1-based) or 0.  mode 0: plain
// FP32 in the oracle's order; 1 / 3: BF16 / split-BF16 trailing updates on the tensor cores.
cudaError_t launch_getrf_large(float *A, int m, int n, int lda, int *ipiv, int *info, LargeStatus *st, int mode,
                               cudaStream_t stream, void *umma_scratch = nullptr);
// Mixed modes: the rank-128 outer updates on tcgen05 tensor cores (lu_large_umma.cu), with
// umma_scratch_bytes(m, n) of device scratch for the operands' BF16 halves.
size_t umma_scratch_bytes(int m, int n);
cudaError_t launch_umma_update(float *A, int lda, int m, int n, int K0, int kend, int bend, int terms,
                               LargeStatus *st, void *scratch, cudaStream_t stream);
// The same in two steps: the BF16 halves of L21 and U12 (columns [bend, n)), then the update
// of columns [c_begin, c_end) within them.
cudaError_t launch_umma_split(float *A, int lda, int m, int n, int K0, int kend, int bend, LargeStatus *st,
                              void *scratch, cudaStream_t stream);
cudaError_t launch_umma_range(float *A, int lda, int m, int n, int kend, int bend, int c_begin, int c_end, int terms,
                              LargeStatus *st, void *scratch, cudaStream_t stream);

// Solve with the factors of launch_getrf_large (or any LAPACK-layout LU) over the whole GPU:
// A is A1 or slot 0 of At, X (n x nrhs, ldx) is X1 or slot 0 of Xt and is overwritten; ipiv
// may be null.  scratch: large_solve_scratch_bytes(n, nrhs) of device memory.  An out-of-range
// pivot sets *bad (device) and leaves X unchanged; info (device, optional) receives -6 then,
// 0 otherwise.  Same per-element order as the oracle's sgetrs.
constexpr int LARGE_SOLVE_MAX_RHS = 16;
size_t large_solve_scratch_bytes(int n, int nrhs);
cudaError_t launch_getrs_large(const float *A1, const float *const *At, int lda, int n, const int *ipiv, float *X1,
                               float *const *Xt, int ldx, int nrhs, void *scratch, int *bad, int *info,
                               cudaStream_t stream, const int *perm_in = nullptr, const float *dinv = nullptr);
// dinv (refinement solves only: not the oracle's order): the inverses of the factors' 128 x 128
// diagonal blocks (large_diag_inverse_bytes(n) of device memory), applied as products.
size_t large_diag_inverse_bytes(int n);
cudaError_t launch_large_diag_inverses(const float *A, int lda, int n, float *inv, cudaStream_t stream);
// perm[i] = the row that ipiv's swaps bring to position i (n ints), for repeated solves
// (perm_in above); *bad as above.
cudaError_t launch_large_perm(const int *ipiv, int n, int *perm, int *bad, cudaStream_t stream);

// ---- refinement of one large matrix (lu_large_refine.cu) ---------------------------------
enum
{
    LIR_RUNNING = 0,
    LIR_CONVERGED = 1,
    LIR_STALLED = 2
};
struct LargeIr
{
    double *x64, *xprev;  // n x nrhs (ld n): the iterate and the one before the last correction
    float *r32;           // n x nrhs: residual, then correction (the solves work in place)
    double *part, *apart;  // per column chunk: partial A x and |A| row sums
    double *bmax, *amax;   // per row block: max |r|, |x|, |b| per right-hand side; max |A| row sum
    double *berr;          // per right-hand side
    int *state, *iters, *take, *running;
};
size_t large_ir_bytes(int n, int nrhs);
LargeIr large_ir_carve(void *base, int n, int nrhs);
cudaError_t launch_lir_init(const LargeIr &s, const float *const *B, int ldb, int n, int nrhs, cudaStream_t st);
cudaError_t launch_lir_update(const LargeIr &s, int n, int nrhs, int first, cudaStream_t st);
cudaError_t launch_lir_residual(const LargeIr &s, const float *const *A, int lda, const float *const *B, int ldb,
                                int n, int nrhs, double tol, int first, cudaStream_t st);
cudaError_t launch_lir_finish(const LargeIr &s, float *const *X, int ldx, int n, int nrhs, double *berr, int *iters,
                              int failed, cudaStream_t st);

// dinv (optional, refinement solves): the diagonal blocks' inverses from
// launch_diag_inverses; the 32 x 32 triangles are then applied as products (not in the
// oracle's order: used where the result is refined, not where it must match bit for bit).
// Inverses above the small orders (tables only): C = A^-1 from LU factors and pivots as the
// blocked solve against the identity; info as the small inverse reports it; scratch:
// getri_blocked_scratch_bytes(n, count).
cudaError_t launch_getri_blocked(const RealBatch &a, const int *ipiv, const RealBatch &c, int *info, void *scratch,
                                 cudaStream_t stream);
size_t getri_blocked_scratch_bytes(int n, int count);
cudaError_t launch_getrs_blocked(const RealBatch &a, const int *ipiv, const int *perm, const RealBatch &b, int nrhs,
                                 int *info, const int *skip, cudaStream_t stream, const float *dinv = nullptr,
                                 const short *lists = nullptr, int trans = 0);
// dinv[(q * nblk + b) * 2 + {0: L, 1: U}] = inverse of the 32 x 32 diagonal block b of the
// factors of matrix q (column-major 32 x 32, nblk = ceil(n / 32)).
cudaError_t launch_diag_inverses(const RealBatch &a, float *dinv, cudaStream_t stream);
// perm[q*n + i] = row of b that the interchanges ipiv[q*n ..] bring to position i.
cudaError_t launch_permutation(const int *ipiv, int *perm, int n, int count, cudaStream_t stream);

// ---- validation and staging ------------------------------------------------------------
// flag[0] |= 1 when any of the m x n leading entries of any matrix is NaN or infinite.
cudaError_t launch_finite_scan(const RealBatch &a, int m, int *flag, cudaStream_t stream);
// dst[i + j*ldd] = src[i + j*lds] for each matrix (copy of the leading m x n block).
cudaError_t launch_copy_matrices(const RealBatch &src, const RealBatch &dst, int m, cudaStream_t stream);
// table[q] = base + q * stride (floats), q < count.
cudaError_t launch_strided_table(float **table, float *base, int64_t stride, int count, cudaStream_t stream);
// dst (column-major, ldd) = transpose of src (column-major, lds), src rows x cols.
cudaError_t launch_transpose(const float *src, int lds, float *dst, int ldd, int rows, int cols,
                             cudaStream_t stream);

}  // namespace ops_solver
