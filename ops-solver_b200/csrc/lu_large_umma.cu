// lu_large_umma.cu -- the large mixed-precision trailing update C -= L21 U12 (K = 128) on the
// fifth-generation tensor cores: tcgen05.mma (kind::f16, BF16 operands from shared memory,
// FP32 accumulator in tensor memory), one elected thread issuing, completion through
// tcgen05.commit on an mbarrier, the accumulator read back with tcgen05.ld.
//
// L21 and U12 are first split into BF16 halves (hi = bf16(v), lo = bf16(v - hi)) in K-major
// workspace arrays (128 values of k per row / column); zero-pivot columns of L are zeroed.
// Each block computes a 128 x 256 tile of C: per 64-wide K chunk the halves of its L21 rows
// and U12 columns are copied (cp.async) into the canonical no-swizzle K-major layout -- core
// matrices of 8 rows x 16 bytes, 8-row groups 256 bytes apart (SBO), the two 8-element halves
// of a 16-wide k step 128 bytes apart (LBO) -- and three products per k step (hi*hi, hi*lo,
// lo*hi) accumulate into the same 128 x 256 FP32 accumulator.
#include <cuda_bf16.h>

#include "common.cuh"
#include "device_once.h"
#include "launch.h"

namespace ops_solver
{
namespace
{
constexpr int UM = 128;        // tile rows (MMA M)
constexpr int UN = 256;        // tile columns (MMA N)
constexpr int UK = 128;        // the update's depth
constexpr int KC = 64;         // k per staged chunk
constexpr int KS = 16;         // k per MMA
constexpr int A_SLAB = UM * KS * 2;  // bytes of one 16-wide k step of A (4 KB)
constexpr int B_SLAB = UN * KS * 2;  // ... of B (8 KB)
constexpr int A_CHUNK = A_SLAB * (KC / KS);
constexpr int B_CHUNK = B_SLAB * (KC / KS);
constexpr int UT = 256;        // threads: warps w and w + 4 share tensor-memory lanes 32 (w % 4)..
constexpr long long UWAIT = 1ll << 20;  // bounded mbarrier wait (try_wait rounds)
constexpr size_t UMMA_SMEM = 2 * (size_t)A_CHUNK + 2 * (size_t)B_CHUNK + 1024;

__device__ __forceinline__ unsigned saddr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, no swizzle, K-major: start, LBO and SBO in 16-byte units,
// descriptor version 1 (bits 46-47), layout type 0.
__device__ __forceinline__ unsigned long long smem_desc(unsigned addr, unsigned lbo, unsigned sbo)
{
    return (unsigned long long)((addr >> 4) & 0x3fffu) | ((unsigned long long)((lbo >> 4) & 0x3fffu) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: F32 accumulator (bits 4-5 = 1), BF16 A and B (bits 7-9
// and 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr unsigned IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(UN >> 3) << 17) | ((unsigned)(UM >> 4) << 24);

__device__ __forceinline__ void umma(unsigned tmem, unsigned long long da, unsigned long long db, unsigned accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(da), "l"(db), "r"(IDESC), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ bool bar_wait(unsigned bar, unsigned parity)
{
    for (long long it = 0; it < UWAIT; ++it)
    {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Split L21 (rows r0.., columns K0..K0+127 of A) into K-major BF16 halves Lh/Ll[row][k].
// (terms 1, BF16 mode, uses the high halves only.)
__global__ void __launch_bounds__(256) umma_split_l(const float *A, int lda, int r0, int rows, int K0,
                                                   const LargeStatus *st, __nv_bfloat16 *Lh, __nv_bfloat16 *Ll)
{
    __shared__ float tile[UK][33];
    const int t = threadIdx.x;
    const int rb = blockIdx.x * 32;  // 32 rows per block
    for (int e = t; e < UK * 32; e += 256)
    {
        const int k = e / 32, r = e % 32;
        const bool zero = (st->zmask[(K0 + k) / 32] >> ((K0 + k) % 32)) & 1u;
        tile[k][r] = (rb + r < rows && !zero) ? A[(int64_t)(K0 + k) * lda + r0 + rb + r] : 0.0f;
    }
    __syncthreads();
    for (int e = t; e < 32 * UK; e += 256)
    {
        const int r = e / UK, k = e % UK;
        if (rb + r >= rows) continue;
        const float v = tile[k][r];
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        Lh[(int64_t)(rb + r) * UK + k] = h;
        Ll[(int64_t)(rb + r) * UK + k] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
}

// Split U12 (rows K0..K0+127, columns c0.. of A) into K-major halves Uh/Ul[col][k].
__global__ void __launch_bounds__(256) umma_split_u(const float *A, int lda, int K0, int c0, int cols,
                                                   __nv_bfloat16 *Uh, __nv_bfloat16 *Ul)
{
    const int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (e >= (int64_t)cols * UK) return;
    const int c = (int)(e / UK), k = (int)(e % UK);
    const float v = A[(int64_t)(c0 + c) * lda + K0 + k];
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    Uh[e] = h;
    Ul[e] = __float2bfloat16_rn(v - __bfloat162float(h));
}

// Copy one K chunk of a tile's operand halves into the canonical layout: nrow rows (row x of
// the tile is global row base + x of the K-major array, valid while < limit), k range
// kc .. kc + 63.  16-byte chunk (x, step s, half h) lands at s * slab + (x / 8) * 256 + h * 128
// + (x % 8) * 16.
__device__ __forceinline__ void stage_operand(unsigned char *dst, int slab, const __nv_bfloat16 *src, int base,
                                              int limit, int nrow, int kc)
{
    const int per = nrow * (KC / 8);  // 16-byte pieces
    for (int e = threadIdx.x; e < per; e += UT)
    {
        const int x = e / (KC / 8), piece = e % (KC / 8);
        const int s = piece / 2, h = piece % 2;
        const unsigned d = saddr(dst + s * slab + (x / 8) * 256 + h * 128 + (x % 8) * 16);
        const bool ok = base + x < limit;
        const __nv_bfloat16 *p = src + (int64_t)(ok ? base + x : 0) * UK + kc + piece * 8;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(p), "r"(ok ? 16 : 0) : "memory");
    }
}

__global__ void __launch_bounds__(UT, 1) umma_update_kernel(float *A, int lda, int r0, int rows, int c0, int cols,
                                                            const __nv_bfloat16 *Lh, const __nv_bfloat16 *Ll,
                                                            const __nv_bfloat16 *Uh, const __nv_bfloat16 *Ul,
                                                            int terms, LargeStatus *st)
{
    extern __shared__ __align__(1024) unsigned char usm[];
    __shared__ unsigned long long bar;
    __shared__ unsigned tmem_base;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    unsigned char *ah = usm, *al = usm + A_CHUNK;
    unsigned char *bh = usm + 2 * A_CHUNK, *bl = bh + B_CHUNK;
    const int rt = blockIdx.x * UM, ct = blockIdx.y * UN;  // tile origin within the update
    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&tmem_base)),
                     "r"(UN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (t == 0)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(&bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = tmem_base;
    bool ok = true;
    for (int c = 0; c < UK / KC; ++c)
    {
        const int kc = c * KC;
        stage_operand(ah, A_SLAB, Lh, rt, rows, UM, kc);
        stage_operand(al, A_SLAB, Ll, rt, rows, UM, kc);
        stage_operand(bh, B_SLAB, Uh, ct, cols, UN, kc);
        stage_operand(bl, B_SLAB, Ul, ct, cols, UN, kc);
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_all;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the copies, visible to the tensor cores
        __syncthreads();
        if (t == 0)
        {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (int s = 0; s < KC / KS; ++s)
            {
                const unsigned long long dah = smem_desc(saddr(ah + s * A_SLAB), 128, 256);
                const unsigned long long dal = smem_desc(saddr(al + s * A_SLAB), 128, 256);
                const unsigned long long dbh = smem_desc(saddr(bh + s * B_SLAB), 128, 256);
                const unsigned long long dbl = smem_desc(saddr(bl + s * B_SLAB), 128, 256);
                umma(tmem, dah, dbh, (c | s) != 0);
                if (terms > 1)
                {
                    umma(tmem, dah, dbl, 1);
                    umma(tmem, dal, dbh, 1);
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             saddr(&bar))
                         : "memory");
        }
        // the chunk's products are done before its shared memory is refilled (or read back)
        if (ok && !bar_wait(saddr(&bar), (unsigned)c & 1u)) ok = false;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    // epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. + 31 (tile rows) for the columns
    // of half w / 4, 32 at a time; each group's C values are all loaded before any is stored
    const int quarter = warp & 3, half = warp >> 2;
    const int row = rt + 32 * quarter + lane;
    const bool rowok = ok && row < rows;
    for (int j = 0; j < UN / 64; ++j)
    {
        const int cb = ct + half * (UN / 2) + 32 * j;  // first column of the group (tile-relative)
        float cv[32];
#pragma unroll
        for (int q = 0; q < 32; ++q)
            cv[q] = (rowok && cb + q < cols) ? A[(int64_t)(c0 + cb + q) * lda + r0 + row] : 0.0f;
        unsigned v[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%"
            "18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
              "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
              "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
              "=r"(v[30]), "=r"(v[31])
            : "r"(tmem + ((unsigned)(32 * quarter) << 16) + (unsigned)(half * (UN / 2) + 32 * j)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (rowok)
        {
#pragma unroll
            for (int q = 0; q < 32; ++q)
                if (cb + q < cols) A[(int64_t)(c0 + cb + q) * lda + r0 + row] = cv[q] - __uint_as_float(v[q]);
        }
    }
    if (!ok && t == 0) st->error = 1;
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(UN) : "memory");
}

}  // namespace

size_t umma_scratch_bytes(int m, int n) { return ((size_t)m + n) * UK * 2 * sizeof(__nv_bfloat16) + 256; }

namespace
{
struct UmmaHalves
{
    __nv_bfloat16 *Lh, *Ll, *Uh, *Ul;
};
UmmaHalves halves(void *scratch, int m, int n)
{
    UmmaHalves h;
    h.Lh = static_cast<__nv_bfloat16 *>(scratch);
    h.Ll = h.Lh + (size_t)m * UK;
    h.Uh = h.Ll + (size_t)m * UK;
    h.Ul = h.Uh + (size_t)n * UK;
    return h;
}
}  // namespace

cudaError_t launch_umma_split(float *A, int lda, int m, int n, int K0, int kend, int bend, LargeStatus *st,
                              void *scratch, cudaStream_t stream)
{
    const int rows = m - kend, cols = n - bend;
    const UmmaHalves h = halves(scratch, m, n);
    umma_split_l<<<(rows + 31) / 32, 256, 0, stream>>>(A, lda, kend, rows, K0, st, h.Lh, h.Ll);
    umma_split_u<<<(unsigned)(((int64_t)cols * UK + 255) / 256), 256, 0, stream>>>(A, lda, K0, bend, cols, h.Uh, h.Ul);
    return cudaGetLastError();
}

cudaError_t launch_umma_range(float *A, int lda, int m, int n, int kend, int bend, int c_begin, int c_end, int terms,
                              LargeStatus *st, void *scratch, cudaStream_t stream)
{
    static std::atomic<unsigned long long> attr{0};
    cudaError_t ea = once_per_device(attr, [] {
        return cudaFuncSetAttribute(umma_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)UMMA_SMEM);
    });
    if (ea != cudaSuccess) return ea;
    const int rows = m - kend, cols = c_end - c_begin;
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    const UmmaHalves h = halves(scratch, m, n);
    const size_t off = (size_t)(c_begin - bend) * UK;  // the range's first column among the split ones
    dim3 g((rows + UM - 1) / UM, (cols + UN - 1) / UN);
    umma_update_kernel<<<g, UT, UMMA_SMEM, stream>>>(A, lda, kend, rows, c_begin, cols, h.Lh, h.Ll, h.Uh + off,
                                                     h.Ul + off, terms, st);
    return cudaGetLastError();
}

cudaError_t launch_umma_update(float *A, int lda, int m, int n, int K0, int kend, int bend, int terms,
                               LargeStatus *st, void *scratch, cudaStream_t stream)
{
    cudaError_t e = launch_umma_split(A, lda, m, n, K0, kend, bend, st, scratch, stream);
    if (e != cudaSuccess) return e;
    return launch_umma_range(A, lda, m, n, kend, bend, bend, n, terms, st, scratch, stream);
}

}  // namespace ops_solver
