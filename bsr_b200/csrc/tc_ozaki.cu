// FP64 product from 8-bit integer digits on the 5th-generation tensor cores
// (tcgen05.mma kind::i8, exact int32 accumulation in tensor memory).
//
// The mixed-precision form of the assembly's direct contraction.  It follows the
// error-free splitting of Ozaki, Ogita, Oishi and Rump ("Error-free transformations
// of matrix multiplication by using fast routines of matrix multiplication and its
// applications", Numer. Algorithms 59, 2012) in its integer form (Mukunoki, Ozaki,
// Ogita, Imamura, "DGEMM using Tensor Cores, and Its Accurate and Reproducible
// Versions", ISC 2020; Ootomo, Ozaki, Yokota 2024 for int8 digits):
//
//   row i of A is scaled by 2^-ea_i (max |a_i.| < 2^ea_i) and column j of B by
//   2^-eb_j, and each scaled value x in (-1, 1) is cut into S signed 7-bit digits,
//   x = sum_t q_t 2^(-7(t+1)) + r, |q_t| <= 127, |r| < 2^(-7S) (every step exact in FP64);
//   C_ij = 2^(ea_i + eb_j) sum_L 2^(-7(L+2)) acc_L(i,j),
//   acc_L = sum_{t+u=L} A_t B_u  (L = 0 .. S-1)  computed exactly in int32.
//
// Every digit product and every int32 sum is exact, so the only errors are the digits
// dropped (terms of order 2^(-7S) of the row and column maxima per K term) and the final
// FP64 sums.  With S = 8 the result agrees with an FP64 GEMM to ~1e-16 K of
// max|a_i.| max|b_.j|.  No counterpart in the reference, which assembles in FP64.
//
// Layout.  A pre-pass writes each operand's digits into a tile image in global memory:
// for every 128-row block of A (64-column block of B) and K step of 32, the S digit
// planes one after another, each plane in the canonical K-major no-swizzle layout of
// the MMA (8-row x 16-byte core matrices; the two 16-byte K halves 128 bytes apart,
// row groups 256 bytes apart).  One stage of the GEMM (one K step, all digits of the
// A block and the B block) is then two contiguous bulk copies (cp.async.bulk, no
// tensor map, no multicast) completed on an mbarrier.
//
// GEMM: one CTA per 128 x 64 tile of C (tiles in groups of 8 row blocks, so CTAs in flight share
// digit blocks in L2), 128 threads, a 4-stage ring in shared memory.
// Thread 0 issues the bulk copies, thread 32 the S(S+1)/2 MMAs (M = 128, N = 64,
// K = 32) of each stage into the S level accumulators (64 TMEM columns each, 512 for
// S = 8) and commits each stage's MMAs to the stage's "empty" mbarrier.  Every wait is
// bounded (2 s of %globaltimer): a wait that runs out sets *err and the CTA drains its
// copies and MMAs (again bounded) before it frees TMEM and returns.  The epilogue reads
// the accumulators with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = rows of C).
#include <cstdint>

#include "bsrg_internal.h"

namespace bsrg {
namespace {

constexpr int OZ_M = 128, OZ_N = 64, OZ_K = 32, OZ_NT = 128;
constexpr int OZ_SMAX = 8;
constexpr int OZ_ASTEP = OZ_M * OZ_K;          // bytes of one digit plane of a 128-row block, one K step
constexpr int OZ_BSTEP = OZ_N * OZ_K;          // ... of a 64-column block of B
constexpr int OZ_NST = 4;                      // stages of the shared-memory ring
constexpr int OZ_KPER = 256;                   // K range of one thread of the exponent pass
constexpr int OZ_GM = 8;                       // row blocks per group of the tile order
constexpr unsigned long long OZ_WAIT_NS = 2000000000ull;
constexpr int OZ_ZERO_EXP = -4000;             // below: an all-zero line (exponents start at 0x80808080)

__device__ __forceinline__ unsigned long long oz_time()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int oz_exp(int e) { return e < OZ_ZERO_EXP ? 0 : e; }

// byte offset of element (row r, k) inside one K step (32 bytes of K) of a K-major 8-bit operand
__device__ __forceinline__ int kmaj8(int r, int k)
{
    return (r >> 3) * 256 + (k >> 4) * 128 + (r & 7) * 16 + (k & 15);
}

__device__ __forceinline__ double oz_elem(const double *X, long ldx, int trans, int r, int k)
{
    return trans ? X[k + (long)r * ldx] : X[r + (long)k * ldx];
}

// ex[r] = max over k of the frexp exponent of |x(r, k)| (max |x(r, .)| < 2^ex[r]); element (r, k) of
// the operand is X[r + k ldx] (trans = 0, the rows of A) or X[k + r ldx] (trans = 1, the columns of B).
// A non-finite element sets *err = 2.
__global__ void oz_exp_kernel(int rows, int K, const double *__restrict__ X, long ldx, int trans, int *ex, int *err)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int k0 = blockIdx.y * OZ_KPER, k1 = min(K, k0 + OZ_KPER);
    if (r >= rows) return;
    double mx = 0.0;
    bool bad = false;
    for (int k = k0; k < k1; k++) {
        const double a = fabs(oz_elem(X, ldx, trans, r, k));
        bad |= !(a <= 1.7976931348623157e308);
        mx = fmax(mx, a);
    }
    if (bad) atomicExch(err, 2);
    if (mx > 0.0 && !bad) {
        int e;
        frexp(mx, &e);
        atomicMax(ex + r, e);
    }
}

// Digits of 16 consecutive k of one row r (rows_pad rows, padding rows and k >= K give zero digits),
// written as 16 bytes into each of the S digit planes of the tile image (blocks of `rb` rows).
__global__ void oz_slice_kernel(int rows, int rows_pad, int K, const double *__restrict__ X, long ldx, int trans,
                                const int *__restrict__ ex, int S, int rb, int kst, int8_t *__restrict__ out)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int kc = blockIdx.y;                       // 16-wide chunk of K
    if (r >= rows_pad) return;
    const int e = r < rows ? oz_exp(ex[r]) : 0;
    double v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int k = kc * 16 + q;
        const double x = (r < rows && k < K) ? oz_elem(X, ldx, trans, r, k) : 0.0;
        v[q] = scalbn(x, -e);                        // |v| < 1, exact
    }
    const int blk = r / rb, rr = r - blk * rb, ks = kc >> 1;
    int8_t *base = out + ((size_t)blk * kst + ks) * (size_t)S * rb * OZ_K + kmaj8(rr, (kc & 1) * 16);
    for (int t = 0; t < S; t++) {
        uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const double y = v[q] * 128.0;           // exact; |y| < 128
            const double d = trunc(y);               // |d| <= 127
            v[q] = y - d;                            // exact, |v| < 1
            w[q >> 2] |= ((uint32_t)(int)d & 0xffu) << (8 * (q & 3));
        }
        *(uint4 *)(base + (size_t)t * rb * OZ_K) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// shared-memory matrix descriptor: no swizzle, K-major, LBO 128 B, SBO 256 B, sm_100 version bits
__device__ __forceinline__ uint64_t oz_desc(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((256u >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor: D S32, A and B signed 8-bit, both K-major, N = 64, M = 128
constexpr uint32_t OZ_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(OZ_N >> 3) << 17) |
                              ((uint32_t)(OZ_M >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t dtmem, uint64_t da, uint64_t db, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
        "l"(da), "l"(db), "r"(OZ_IDESC), "r"(accumulate));
}

__device__ __forceinline__ bool mb_wait(uint32_t bar, uint32_t parity)
{
    const unsigned long long t0 = oz_time();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (oz_time() - t0 > OZ_WAIT_NS) return false;
    }
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

template <int S>
__global__ void __launch_bounds__(OZ_NT, 1) oz_gemm_kernel(int M, int N, int kst, int mblk, int nblk, double alpha,
                                                          const int8_t *__restrict__ Asl,
                                                          const int8_t *__restrict__ Bsl, const int *__restrict__ ea,
                                                          const int *__restrict__ eb, double beta, double *C, long ldc,
                                                          int *err)
{
    extern __shared__ __align__(1024) unsigned char osm[];
    constexpr int STAGE = S * (OZ_ASTEP + OZ_BSTEP);
    uint64_t *full = (uint64_t *)(osm + OZ_NST * STAGE);
    uint64_t *empty = full + OZ_NST;
    uint64_t *done = empty + OZ_NST;
    uint32_t *taddr_s = (uint32_t *)(done + 1);
    volatile int *fail_s = (volatile int *)(taddr_s + 1);
    volatile int *issued_s = fail_s + 1;           // stages whose copies were issued
    volatile int *used_s = fail_s + 2;             // stages whose MMAs were issued
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // tile order: groups of OZ_GM row blocks, walked column block by column block, so that the CTAs
    // in flight share a few blocks of A's and B's digits in L2
    const int per = OZ_GM * nblk, grp = (int)blockIdx.x / per, m0b = grp * OZ_GM;
    const int gs = min(mblk - m0b, OZ_GM), rr = (int)blockIdx.x - grp * per;
    const int mb = m0b + rr % gs, nb = rr / gs;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(osm);
    const uint32_t full_a = (uint32_t)__cvta_generic_to_shared(full);
    const uint32_t empty_a = (uint32_t)__cvta_generic_to_shared(empty);
    const uint32_t done_a = (uint32_t)__cvta_generic_to_shared(done);
    if (tid == 0) {
        for (int b = 0; b < OZ_NST; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(full_a + 8 * b));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(empty_a + 8 * b));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(done_a));
        asm volatile("fence.mbarrier_init.release.cluster;" ::);
        *fail_s = 0;
        *issued_s = 0;
        *used_s = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(taddr_s)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
    const uint32_t dtmem = *taddr_s;

    if (tid == 0) {
        // ---- producer: the digit planes of the A block and the B block of each K step ----
        const int8_t *Ab = Asl + (size_t)mb * kst * S * OZ_ASTEP;
        const int8_t *Bb = Bsl + (size_t)nb * kst * S * OZ_BSTEP;
        for (int kt = 0; kt < kst; kt++) {
            const int b = kt % OZ_NST;
            if (kt >= OZ_NST && !mb_wait(empty_a + 8 * b, (uint32_t)((kt / OZ_NST) - 1) & 1u)) {
                *fail_s = 1;
                break;
            }
            if (*fail_s) break;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(full_a + 8 * b),
                         "r"((uint32_t)STAGE)
                         : "memory");
            const uint32_t dst = sbase + (uint32_t)(b * STAGE);
            bulk_g2s(dst, Ab + (size_t)kt * S * OZ_ASTEP, S * OZ_ASTEP, full_a + 8 * b);
            bulk_g2s(dst + S * OZ_ASTEP, Bb + (size_t)kt * S * OZ_BSTEP, S * OZ_BSTEP, full_a + 8 * b);
            *issued_s = kt + 1;
        }
    } else if (tid == 32) {
        // ---- MMA issuer: level L = t + u of the digit products into accumulator L ----
        int kt = 0;
        for (; kt < kst; kt++) {
            const int b = kt % OZ_NST;
            if (!mb_wait(full_a + 8 * b, (uint32_t)(kt / OZ_NST) & 1u)) {
                *fail_s = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::);
            const uint32_t a0 = sbase + (uint32_t)(b * STAGE), b0 = a0 + S * OZ_ASTEP;
#pragma unroll
            for (int t = 0; t < S; t++)
#pragma unroll
                for (int u = 0; u + t < S; u++)
                    mma_i8(dtmem + (uint32_t)((t + u) * OZ_N), oz_desc(a0 + t * OZ_ASTEP), oz_desc(b0 + u * OZ_BSTEP),
                           (kt > 0 || t > 0) ? 1u : 0u);
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             empty_a + 8 * b)
                         : "memory");
            if (*fail_s) { kt++; break; }
        }
        *used_s = kt;
        // arrives once every MMA issued above has completed
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(done_a)
                     : "memory");
    }
    const bool waited = mb_wait(done_a, 0u);
    const bool ok = __syncthreads_and(waited) && !*fail_s;     // uniform over the CTA
    if (!ok) {
        // drain: the MMAs in flight and the copies issued but never consumed finish before TMEM is
        // freed and the CTA leaves
        if (tid == 0) {
            atomicExch(err, 1);
            if (!waited) mb_wait(done_a, 0u);
            const int used = *used_s, issued = *issued_s;
            for (int kt = used; kt < issued; kt++) mb_wait(full_a + 8 * (kt % OZ_NST), (uint32_t)(kt / OZ_NST) & 1u);
        }
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::);
        const int row = mb * OZ_M + warp * 32 + lane;
        const int er = row < M ? oz_exp(ea[row]) : 0;
        const uint32_t tl = dtmem + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < OZ_N; c0 += 8) {
            uint32_t v[S][8];
#pragma unroll
            for (int L = 0; L < S; L++)
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                             : "=r"(v[L][0]), "=r"(v[L][1]), "=r"(v[L][2]), "=r"(v[L][3]), "=r"(v[L][4]),
                               "=r"(v[L][5]), "=r"(v[L][6]), "=r"(v[L][7])
                             : "r"(tl + (uint32_t)(L * OZ_N + c0)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < M) {
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const int col = nb * OZ_N + c0 + j;
                    if (col < N) {
                        double s = 0.0;
#pragma unroll
                        for (int L = S - 1; L >= 0; L--) s += scalbn((double)(int)v[L][j], -7 * (L + 2));
                        double *cp = C + row + (long)col * ldc;
                        double r = alpha * scalbn(s, er + oz_exp(eb[col]));
                        if (beta != 0.0) r += beta * *cp;
                        *cp = r;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(dtmem), "r"(512));
}

__global__ void oz_scale_kernel(int M, int N, double beta, double *C, long ldc)
{
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long)M * N) return;
    double *cp = C + q % M + (q / M) * ldc;
    *cp = beta == 0.0 ? 0.0 : beta * *cp;
}

struct OzLayout {
    size_t kst, mp, np, a_bytes, b_bytes, total;
};

OzLayout oz_layout(int m, int n, int k, int S)
{
    OzLayout L;
    L.kst = ((size_t)k + OZ_K - 1) / OZ_K;
    L.mp = ((size_t)m + OZ_M - 1) / OZ_M * OZ_M;
    L.np = ((size_t)n + OZ_N - 1) / OZ_N * OZ_N;
    L.a_bytes = (size_t)S * L.mp * L.kst * OZ_K;
    L.b_bytes = (size_t)S * L.np * L.kst * OZ_K;
    L.total = L.a_bytes + L.b_bytes + sizeof(int) * (L.mp + L.np) + 256;
    return L;
}

template <int S> int oz_launch(int mblk, int nblk, int m, int n, int kst, double alpha, const int8_t *As,
                               const int8_t *Bs, const int *ea, const int *eb, double beta, double *C, long ldc,
                               int *err, cudaStream_t s)
{
    const int smem = OZ_NST * S * (OZ_ASTEP + OZ_BSTEP) + 128;
    cudaError_t e = smem_attr(oz_gemm_kernel<S>, smem);
    if (e != cudaSuccess) return cuda_fail(e, "ozaki gemm smem");
    oz_gemm_kernel<S><<<(unsigned)(mblk * nblk), OZ_NT, smem, s>>>(m, n, kst, mblk, nblk, alpha, As, Bs, ea, eb, beta,
                                                                   C, ldc, err);
    return cuda_fail(cudaGetLastError(), "ozaki gemm");
}

}  // namespace

size_t ozaki_ws_bytes(int m, int n, int k, int slices)
{
    if (slices <= 0) slices = OZ_SMAX;
    return oz_layout(m, n, k, slices).total;
}

int ozaki_gemm(int m, int n, int k, double alpha, const double *A, long lda, const double *B, long ldb, double beta,
               double *C, long ldc, int slices, void *ws, size_t ws_bytes, int *err, cudaStream_t s)
{
    if (slices <= 0) slices = OZ_SMAX;
    if (slices < 6 || slices > OZ_SMAX) {
        set_error("dgemm_ozaki: slices = %d outside 6..%d", slices, OZ_SMAX);
        return BSRG_ERR_ARG;
    }
    if (k > BSRG_OZAKI_KMAX) {
        set_error("dgemm_ozaki: k = %d above %d (the int32 accumulators could overflow)", k, BSRG_OZAKI_KMAX);
        return BSRG_ERR_ARG;
    }
    if (m <= 0 || n <= 0) return BSRG_OK;
    if (k == 0 || alpha == 0.0) {
        const long mn = (long)m * n;
        oz_scale_kernel<<<(unsigned)((mn + 255) / 256), 256, 0, s>>>(m, n, beta, C, ldc);
        return cuda_fail(cudaGetLastError(), "ozaki gemm (scale)");
    }
    const OzLayout L = oz_layout(m, n, k, slices);
    if (!ws || ws_bytes < L.total || ((uintptr_t)ws & 255)) {
        set_error("dgemm_ozaki: workspace of %zu bytes at %p, %zu bytes (256-byte aligned) needed", ws_bytes, ws,
                  L.total);
        return BSRG_ERR_ARG;
    }
    int8_t *As = (int8_t *)ws, *Bs = As + L.a_bytes;
    int *ea = (int *)(Bs + L.b_bytes), *eb = ea + L.mp;
    cudaError_t e = cudaMemsetAsync(ea, 0x80, sizeof(int) * (L.mp + L.np), s);
    if (e != cudaSuccess) return cuda_fail(e, "ozaki exponents");
    const unsigned kparts = (unsigned)((k + OZ_KPER - 1) / OZ_KPER);
    oz_exp_kernel<<<dim3((unsigned)((m + 127) / 128), kparts), 128, 0, s>>>(m, k, A, lda, 0, ea, err);
    oz_exp_kernel<<<dim3((unsigned)((n + 127) / 128), kparts), 128, 0, s>>>(n, k, B, ldb, 1, eb, err);
    const unsigned kc = (unsigned)(2 * L.kst);
    oz_slice_kernel<<<dim3((unsigned)(L.mp / 128), kc), 128, 0, s>>>(m, (int)L.mp, k, A, lda, 0, ea, slices, OZ_M,
                                                                     (int)L.kst, As);
    oz_slice_kernel<<<dim3((unsigned)((L.np + 127) / 128), kc), 128, 0, s>>>(n, (int)L.np, k, B, ldb, 1, eb, slices,
                                                                             OZ_N, (int)L.kst, Bs);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "ozaki digits");
    const int mblk = (int)(L.mp / OZ_M), nblk = (int)(L.np / OZ_N);
    switch (slices) {
    case 6: return oz_launch<6>(mblk, nblk, m, n, (int)L.kst, alpha, As, Bs, ea, eb, beta, C, ldc, err, s);
    case 7: return oz_launch<7>(mblk, nblk, m, n, (int)L.kst, alpha, As, Bs, ea, eb, beta, C, ldc, err, s);
    default: return oz_launch<8>(mblk, nblk, m, n, (int)L.kst, alpha, As, Bs, ea, eb, beta, C, ldc, err, s);
    }
}

}  // namespace bsrg

using namespace bsrg;

extern "C" size_t bsrg_dgemm_ozaki_work_bytes(int m, int n, int k, int slices)
{
    if (m <= 0 || n <= 0 || k <= 0) return 256;
    return ozaki_ws_bytes(m, n, k, slices);
}

extern "C" int bsrg_dgemm_ozaki(int m, int n, int k, double alpha, const double *A, int lda, const double *B, int ldb,
                                double beta, double *C, int ldc, int slices, void *work, size_t work_bytes, int *err,
                                void *stream)
{
    if ((m > 0 && n > 0) && (!C || !err || (k > 0 && (!A || !B)))) {
        set_error("dgemm_ozaki: null argument");
        return BSRG_ERR_ARG;
    }
    if (m < 0 || n < 0 || k < 0 || lda < (m > 0 ? m : 1) || ldb < (k > 0 ? k : 1) || ldc < (m > 0 ? m : 1)) {
        set_error("dgemm_ozaki: bad sizes m=%d n=%d k=%d lda=%d ldb=%d ldc=%d", m, n, k, lda, ldb, ldc);
        return BSRG_ERR_ARG;
    }
    return ozaki_gemm(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, slices, work, work_bytes, err,
                      (cudaStream_t)stream);
}
