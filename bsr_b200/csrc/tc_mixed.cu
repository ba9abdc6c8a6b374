// Split-precision GEMM on the 5th-generation tensor cores (tcgen05, kind::tf32).
//
// The mixed-precision form of the assembly contractions: FP64 operands are split
// into two TF32 parts, x = hi + lo (hi = x rounded to TF32, lo = the FP64
// remainder rounded to TF32), and C = alpha (Ahi Bhi + Ahi Blo + Alo Bhi) + beta C
// is accumulated in FP32 in tensor memory (TMEM) -- about 22 significant bits per
// operand, FP32 accumulation.  No counterpart in the reference, which assembles
// in FP64; the FP64 path stays the drop-in.
//
// One CTA per 128 x 128 tile of C, 128 threads.  Per K slice of 32: all threads
// convert and store the slices of A and B into shared memory in the canonical
// K-major layout without swizzle (8-row x 16-byte core matrices; the two 16-byte
// K halves of an MMA 128 bytes apart (LBO), row groups 256 bytes apart (SBO));
// one thread issues 3 x 4 tcgen05.mma (M = 128, N = 128, K = 8) into the same
// accumulator and commits them to an mbarrier that every thread waits on (bounded)
// before the slice is overwritten.  The epilogue reads the accumulator with
// tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = rows of C).
#include <cstdint>

#include "bsrg_internal.h"

namespace bsrg {
namespace {

constexpr int TC_M = 128, TC_N = 128, TC_K = 32, TC_NT = 128;
constexpr int TC_KSTEP_BYTES = TC_M * 8 * 4;                 // one K = 8 slice of a 128-row operand (4 KB)
constexpr int TC_OPER_BYTES = TC_KSTEP_BYTES * (TC_K / 8);    // one 128 x 32 TF32 operand slice (16 KB)
constexpr int TC_SMEM = 4 * TC_OPER_BYTES + 64;               // Ahi, Alo, Bhi, Blo + mbarrier + TMEM address
constexpr unsigned long long TC_WAIT_NS = 2000000000ull;

__device__ __forceinline__ unsigned long long tc_time()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// byte offset of element (row r, k) of a 128 x 32 K-major operand slice
__device__ __forceinline__ int kmaj_off(int r, int k)
{
    return (k >> 3) * TC_KSTEP_BYTES + (r >> 3) * 256 + ((k >> 2) & 1) * 128 + (r & 7) * 16 + (k & 3) * 4;
}

__device__ __forceinline__ uint32_t to_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// shared-memory matrix descriptor: no swizzle, K-major, LBO 128 B, SBO 256 B, sm_100 version bits
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((256u >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor: D FP32, A and B TF32, both K-major, N = 128, M = 128
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t da, uint64_t db, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
        "l"(da), "l"(db), "r"(TC_IDESC), "r"(accumulate));
}

__global__ void __launch_bounds__(TC_NT) tf32x3_gemm_kernel(int M, int N, int K, double alpha,
                                                            const double *__restrict__ A, long lda,
                                                            const double *__restrict__ B, long ldb, double beta,
                                                            double *C, long ldc, int *err)
{
    extern __shared__ __align__(1024) unsigned char tsm[];
    unsigned char *Ahi = tsm, *Alo = tsm + TC_OPER_BYTES, *Bhi = tsm + 2 * TC_OPER_BYTES,
                  *Blo = tsm + 3 * TC_OPER_BYTES;
    uint64_t *mbar = (uint64_t *)(tsm + 4 * TC_OPER_BYTES);
    uint32_t *taddr_s = (uint32_t *)(tsm + 4 * TC_OPER_BYTES + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * TC_M, n0 = blockIdx.y * TC_N;
    const uint32_t mbar_a = (uint32_t)__cvta_generic_to_shared(mbar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_a));
        asm volatile("fence.mbarrier_init.release.cluster;" ::);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(taddr_s)),
                     "r"(TC_N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
    const uint32_t dtmem = *taddr_s;
    const int ktiles = (K + TC_K - 1) / TC_K;
    uint32_t phase = 0;
    bool failed = false;
    for (int kt = 0; kt < ktiles; kt++) {
        const int k0 = kt * TC_K;
        // ---- stage the slices: A rows m0.., B columns n0.., split into TF32 parts ----
        for (int q = tid; q < TC_M * TC_K; q += TC_NT) {
            const int r = q % TC_M, k = q / TC_M;          // consecutive threads: consecutive rows of A
            const int gm = m0 + r, gk = k0 + k;
            const double x = (gm < M && gk < K) ? A[gm + (long)gk * lda] : 0.0;
            const uint32_t hi = to_tf32((float)x);
            const uint32_t lo = to_tf32((float)(x - (double)__uint_as_float(hi)));
            const int o = kmaj_off(r, k);
            *(uint32_t *)(Ahi + o) = hi;
            *(uint32_t *)(Alo + o) = lo;
        }
        for (int q = tid; q < TC_N * TC_K; q += TC_NT) {
            const int k = q % TC_K, c = q / TC_K;          // consecutive threads: consecutive k of a column of B
            const int gn = n0 + c, gk = k0 + k;
            const double x = (gn < N && gk < K) ? B[gk + (long)gn * ldb] : 0.0;
            const uint32_t hi = to_tf32((float)x);
            const uint32_t lo = to_tf32((float)(x - (double)__uint_as_float(hi)));
            const int o = kmaj_off(c, k);
            *(uint32_t *)(Bhi + o) = hi;
            *(uint32_t *)(Blo + o) = lo;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // generic writes -> tensor-core reads
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::);
            const uint32_t ah = (uint32_t)__cvta_generic_to_shared(Ahi), al = (uint32_t)__cvta_generic_to_shared(Alo);
            const uint32_t bh = (uint32_t)__cvta_generic_to_shared(Bhi), bl = (uint32_t)__cvta_generic_to_shared(Blo);
#pragma unroll
            for (int s = 0; s < TC_K / 8; s++) {
                const uint32_t off = s * TC_KSTEP_BYTES;
                mma_tf32(dtmem, smem_desc(ah + off), smem_desc(bh + off), (kt > 0 || s > 0) ? 1u : 0u);
                mma_tf32(dtmem, smem_desc(ah + off), smem_desc(bl + off), 1u);
                mma_tf32(dtmem, smem_desc(al + off), smem_desc(bh + off), 1u);
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar_a)
                         : "memory");
        }
        // every thread waits for the MMAs of this slice before the buffers are reused
        {
            const unsigned long long t0 = tc_time();
            uint32_t done = 0;
            while (!done) {
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                    "selp.u32 %0, 1, 0, p;\n\t}\n"
                    : "=r"(done)
                    : "r"(mbar_a), "r"(phase));
                if (!done && tc_time() - t0 > TC_WAIT_NS) { failed = true; break; }
            }
        }
        phase ^= 1u;
        if (__syncthreads_or(failed)) { failed = true; break; }
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
    if (failed) {
        if (tid == 0) atomicExch(err, 1);
    } else if (ktiles > 0) {
        // ---- epilogue: warp w reads TMEM lanes 32w.. (rows), 8 columns at a time ----
        const int row = m0 + warp * 32 + lane;
        for (int c0 = 0; c0 < TC_N; c0 += 8) {
            uint32_t v[8];
            const uint32_t ta = dtmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7])
                         : "r"(ta));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < M)
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const int col = n0 + c0 + j;
                    if (col < N) {
                        double *cp = C + row + (long)col * ldc;
                        double r = alpha * (double)__uint_as_float(v[j]);
                        if (beta != 0.0) r += beta * *cp;
                        *cp = r;
                    }
                }
        }
    } else {
        // K = 0: C = beta C
        for (int q = tid; q < TC_M * TC_N; q += TC_NT) {
            const int r = m0 + q % TC_M, col = n0 + q / TC_M;
            if (r < M && col < N) C[r + (long)col * ldc] *= beta;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(dtmem), "r"(TC_N));
}

}  // namespace

int tf32x3_gemm(int m, int n, int k, double alpha, const double *A, long lda, const double *B, long ldb, double beta,
                double *C, long ldc, int *err, cudaStream_t s)
{
    if (m <= 0 || n <= 0) return BSRG_OK;
    cudaError_t e = smem_attr(tf32x3_gemm_kernel, TC_SMEM);
    if (e != cudaSuccess) return cuda_fail(e, "tf32x3 gemm smem");
    dim3 g((unsigned)((m + TC_M - 1) / TC_M), (unsigned)((n + TC_N - 1) / TC_N));
    tf32x3_gemm_kernel<<<g, TC_NT, TC_SMEM, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, err);
    return cuda_fail(cudaGetLastError(), "tf32x3 gemm");
}

}  // namespace bsrg

using namespace bsrg;

extern "C" int bsrg_dgemm_tf32x3(int m, int n, int k, double alpha, const double *A, int lda, const double *B,
                                 int ldb, double beta, double *C, int ldc, int *err, void *stream)
{
    if ((m > 0 && n > 0) && (!C || !err || (k > 0 && (!A || !B)))) {
        set_error("dgemm_tf32x3: null argument");
        return BSRG_ERR_ARG;
    }
    if (m < 0 || n < 0 || k < 0 || lda < (m > 0 ? m : 1) || ldb < (k > 0 ? k : 1) || ldc < (m > 0 ? m : 1)) {
        set_error("dgemm_tf32x3: bad sizes m=%d n=%d k=%d lda=%d ldb=%d ldc=%d", m, n, k, lda, ldb, ldc);
        return BSRG_ERR_ARG;
    }
    return tf32x3_gemm(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, err, (cudaStream_t)stream);
}
