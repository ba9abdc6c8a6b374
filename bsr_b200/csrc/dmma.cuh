// FP64 tensor-core GEMM core for sm_100a: mma.sync.aligned.m8n8k4 f64 (DMMA).
//
// FP64 has no tcgen05 kind, so the FP64 tensor pipe is reached through the
// warp-level m8n8k4 f64 MMA.  One CTA computes a 128 x 128 tile of
// C = op(A) op(B) with 8 warps (2 along M x 4 along N, 64 x 32 per warp:
// 8 x 4 MMA tiles, 64 accumulators per thread).  K advances in steps of 16
// through a 3-stage cp.async pipeline; every operand tile is staged in shared
// memory in the orientation its global layout gives (no transposes), with a
// padding of 4 doubles so that the fragment loads of each half-warp hit 16
// distinct 8-byte bank slots.
//
// Fragment layouts of m8n8k4 f64 (row.col): A 8x4 -- lane holds A[lane>>2][lane&3];
// B 4x8 -- lane holds B[lane&3][lane>>2]; C 8x8 -- lane holds C[lane>>2][2(lane&3)+{0,1}].
//
// All matrices are column-major (Fortran).  op(A) is M x K: A (lda >= M) when
// TA is false, A^T of a K x M array when TA is true; likewise op(B) is K x N.
#pragma once
#include <cuda_runtime.h>

namespace bsrg {
namespace dmma {

constexpr int BM = 128, BN = 128, BK = 16, STAGES = 3, NT = 256;
constexpr int PAD = 4;

template <bool TA> struct ALayout {
    // !TA: As[k][m] (m contiguous), TA: As[m][k] (k contiguous)
    static constexpr int ELEMS = TA ? BM * (BK + PAD) : BK * (BM + PAD);
};
template <bool TB> struct BLayout {
    // !TB: Bs[n][k] (k contiguous), TB: Bs[k][n] (n contiguous)
    static constexpr int ELEMS = TB ? BK * (BN + PAD) : BN * (BK + PAD);
};

template <bool TA, bool TB> struct Smem {
    static constexpr int STAGE = ALayout<TA>::ELEMS + BLayout<TB>::ELEMS;
    static constexpr int BYTES = STAGES * STAGE * 8;
};

__device__ __forceinline__ void cp_async8(double *smem, const double *gmem, bool valid)
{
    unsigned saddr = (unsigned)__cvta_generic_to_shared(smem);
    int bytes = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void mma884(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// stage one BK slice of the A and B tiles (zero-filled outside the matrices)
template <bool TA, bool TB>
__device__ __forceinline__ void load_stage(double *sA, double *sB, const double *A, long lda, const double *B,
                                           long ldb, int M, int N, int K, int m0, int n0, int k0)
{
    const int tid = threadIdx.x;
#pragma unroll
    for (int i = 0; i < (BM * BK) / NT; i++) {
        const int idx = tid + i * NT;
        int ml, kl;
        if (!TA) { ml = idx % BM; kl = idx / BM; }
        else { kl = idx % BK; ml = idx / BK; }
        const int gm = m0 + ml, gk = k0 + kl;
        const bool v = gm < M && gk < K;
        const double *src = v ? (TA ? A + gk + (long)gm * lda : A + gm + (long)gk * lda) : A;
        double *dst = TA ? sA + ml * (BK + PAD) + kl : sA + kl * (BM + PAD) + ml;
        cp_async8(dst, src, v);
    }
#pragma unroll
    for (int i = 0; i < (BN * BK) / NT; i++) {
        const int idx = tid + i * NT;
        int nl, kl;
        if (!TB) { kl = idx % BK; nl = idx / BK; }
        else { nl = idx % BN; kl = idx / BN; }
        const int gn = n0 + nl, gk = k0 + kl;
        const bool v = gn < N && gk < K;
        const double *src = v ? (TB ? B + gn + (long)gk * ldb : B + gk + (long)gn * ldb) : B;
        double *dst = TB ? sB + kl * (BN + PAD) + nl : sB + nl * (BK + PAD) + kl;
        cp_async8(dst, src, v);
    }
}

// acc[s][t][j]: row m0 + wm*64 + s*8 + (lane>>2), column n0 + wn*32 + t*8 + 2*(lane&3) + j
template <bool TA, bool TB>
__device__ __forceinline__ void tile_mma(double acc[8][4][2], double *smem, const double *A, long lda,
                                         const double *B, long ldb, int M, int N, int K, int m0, int n0)
{
    constexpr int SA = ALayout<TA>::ELEMS, STG = Smem<TA, TB>::STAGE;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm = warp & 1, wn = warp >> 1;
    const int r = lane >> 2, c = lane & 3;
#pragma unroll
    for (int s = 0; s < 8; s++)
#pragma unroll
        for (int t = 0; t < 4; t++) acc[s][t][0] = acc[s][t][1] = 0.0;
    const int ktiles = (K + BK - 1) / BK;
#pragma unroll
    for (int st = 0; st < STAGES - 1; st++) {
        if (st < ktiles)
            load_stage<TA, TB>(smem + st * STG, smem + st * STG + SA, A, lda, B, ldb, M, N, K, m0, n0, st * BK);
        cp_async_commit();
    }
    for (int kt = 0; kt < ktiles; kt++) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        const int nk = kt + STAGES - 1;
        if (nk < ktiles) {
            double *base = smem + (nk % STAGES) * STG;
            load_stage<TA, TB>(base, base + SA, A, lda, B, ldb, M, N, K, m0, n0, nk * BK);
        }
        cp_async_commit();
        const double *sA = smem + (kt % STAGES) * STG, *sB = sA + SA;
#pragma unroll
        for (int kk = 0; kk < BK / 4; kk++) {
            double af[8], bf[4];
#pragma unroll
            for (int s = 0; s < 8; s++) {
                const int ml = wm * 64 + s * 8 + r, kl = kk * 4 + c;
                af[s] = TA ? sA[ml * (BK + PAD) + kl] : sA[kl * (BM + PAD) + ml];
            }
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const int nl = wn * 32 + t * 8 + r, kl = kk * 4 + c;
                bf[t] = TB ? sB[kl * (BN + PAD) + nl] : sB[nl * (BK + PAD) + kl];
            }
#pragma unroll
            for (int s = 0; s < 8; s++)
#pragma unroll
                for (int t = 0; t < 4; t++) mma884(acc[s][t][0], acc[s][t][1], af[s], bf[t]);
        }
    }
    cp_async_wait<0>();
    __syncthreads();
}

}  // namespace dmma
}  // namespace bsrg
