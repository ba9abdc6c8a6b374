// FP64 tensor-core GEMM core for sm_100a: mma.sync.aligned.m8n8k4 f64 (DMMA).
//
// FP64 has no tcgen05 kind, so the FP64 tensor pipe is reached through the
// warp-level m8n8k4 f64 MMA.  A CTA computes a BM x BN tile of
// C = op(A) op(B) with WM x WN warps, each warp a (BM/WM) x (BN/WN) sub-tile of
// 8 x 8 MMA tiles.  K advances in steps of 16 through a 3-stage cp.async
// pipeline; every operand tile is staged in shared memory in the orientation
// its global layout gives (no transposes), with a padding of 4 doubles so that
// the fragment loads of each half-warp hit 16 distinct 8-byte bank slots.
// Shapes: 128 x 128 (8 warps, 64 x 32 each) for square work, 128 x 32 and
// 32 x 128 (4 warps, 32 x 32 each) for the panel products of the eigensolver.
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

constexpr int BK = 16, STAGES = 3, PAD = 4;

template <int BM_, int BN_, int WM_, int WN_> struct Cfg {
    static constexpr int BM = BM_, BN = BN_, WM = WM_, WN = WN_;
    static constexpr int NT = 32 * WM * WN;
    static constexpr int TM = BM / WM, TN = BN / WN;     // warp tile
    static constexpr int FM = TM / 8, FN = TN / 8;       // MMA tiles per warp
    static_assert(TM % 8 == 0 && TN % 8 == 0, "warp tile of whole 8x8 MMA tiles");
    static_assert((BM * BK) % NT == 0 && (BN * BK) % NT == 0, "whole loads per thread");
};
using Sq = Cfg<128, 128, 2, 4>;   // 256 threads
using Tall = Cfg<128, 32, 4, 1>;  // 128 threads
using Wide = Cfg<32, 128, 1, 4>;  // 128 threads

template <class C, bool TA> struct ALayout {
    // !TA: As[k][m] (m contiguous), TA: As[m][k] (k contiguous)
    static constexpr int ELEMS = TA ? C::BM * (BK + PAD) : BK * (C::BM + PAD);
};
template <class C, bool TB> struct BLayout {
    // !TB: Bs[n][k] (k contiguous), TB: Bs[k][n] (n contiguous)
    static constexpr int ELEMS = TB ? BK * (C::BN + PAD) : C::BN * (BK + PAD);
};
template <class C, bool TA, bool TB> struct Smem {
    static constexpr int STAGE = ALayout<C, TA>::ELEMS + BLayout<C, TB>::ELEMS;
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

// stage one BK slice of the A and B tiles (zero-filled outside the matrices and
// outside the K range [k0, kend)).  SYMA: A is square symmetric with only its lower
// triangle stored; element (m, k) is read from (max, min), a tile wholly above the
// diagonal with the index order that keeps the reads coalesced.
template <class C, bool TA, bool TB, bool SYMA = false>
__device__ __forceinline__ void load_stage(double *sA, double *sB, const double *A, long lda, const double *B,
                                           long ldb, int M, int N, int kend, int m0, int n0, int k0)
{
    const int tid = threadIdx.x;
    const bool upper_tile = SYMA && m0 + C::BM <= k0;
#pragma unroll
    for (int i = 0; i < (C::BM * BK) / C::NT; i++) {
        const int idx = tid + i * C::NT;
        int ml, kl;
        if (!TA && !upper_tile) { ml = idx % C::BM; kl = idx / C::BM; }
        else { kl = idx % BK; ml = idx / BK; }
        const int gm = m0 + ml, gk = k0 + kl;
        const bool v = gm < M && gk < kend;
        const double *src;
        if (SYMA) src = v ? (gm >= gk ? A + gm + (long)gk * lda : A + gk + (long)gm * lda) : A;
        else src = v ? (TA ? A + gk + (long)gm * lda : A + gm + (long)gk * lda) : A;
        double *dst = TA ? sA + ml * (BK + PAD) + kl : sA + kl * (C::BM + PAD) + ml;
        cp_async8(dst, src, v);
    }
#pragma unroll
    for (int i = 0; i < (C::BN * BK) / C::NT; i++) {
        const int idx = tid + i * C::NT;
        int nl, kl;
        if (!TB) { kl = idx % BK; nl = idx / BK; }
        else { nl = idx % C::BN; kl = idx / C::BN; }
        const int gn = n0 + nl, gk = k0 + kl;
        const bool v = gn < N && gk < kend;
        const double *src = v ? (TB ? B + gn + (long)gk * ldb : B + gk + (long)gn * ldb) : B;
        double *dst = TB ? sB + kl * (C::BN + PAD) + nl : sB + nl * (BK + PAD) + kl;
        cp_async8(dst, src, v);
    }
}

// acc[s][t][j]: row m0 + wm*TM + s*8 + (lane>>2), column n0 + wn*TN + t*8 + 2*(lane&3) + j,
// summed over k in [kbeg, kend)
template <class C, bool TA, bool TB, bool SYMA = false>
__device__ __forceinline__ void tile_mma(double (&acc)[C::FM][C::FN][2], double *smem, const double *A, long lda,
                                         const double *B, long ldb, int M, int N, int kbeg, int kend, int m0, int n0)
{
    constexpr int SA = ALayout<C, TA>::ELEMS, STG = Smem<C, TA, TB>::STAGE;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm = warp % C::WM, wn = warp / C::WM;
    const int r = lane >> 2, c = lane & 3;
#pragma unroll
    for (int s = 0; s < C::FM; s++)
#pragma unroll
        for (int t = 0; t < C::FN; t++) acc[s][t][0] = acc[s][t][1] = 0.0;
    const int ktiles = kend > kbeg ? (kend - kbeg + BK - 1) / BK : 0;
#pragma unroll
    for (int st = 0; st < STAGES - 1; st++) {
        if (st < ktiles)
            load_stage<C, TA, TB, SYMA>(smem + st * STG, smem + st * STG + SA, A, lda, B, ldb, M, N, kend, m0, n0,
                                        kbeg + st * BK);
        cp_async_commit();
    }
    for (int kt = 0; kt < ktiles; kt++) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        const int nk = kt + STAGES - 1;
        if (nk < ktiles) {
            double *base = smem + (nk % STAGES) * STG;
            load_stage<C, TA, TB, SYMA>(base, base + SA, A, lda, B, ldb, M, N, kend, m0, n0, kbeg + nk * BK);
        }
        cp_async_commit();
        const double *sA = smem + (kt % STAGES) * STG, *sB = sA + SA;
#pragma unroll
        for (int kk = 0; kk < BK / 4; kk++) {
            double af[C::FM], bf[C::FN];
#pragma unroll
            for (int s = 0; s < C::FM; s++) {
                const int ml = wm * C::TM + s * 8 + r, kl = kk * 4 + c;
                af[s] = TA ? sA[ml * (BK + PAD) + kl] : sA[kl * (C::BM + PAD) + ml];
            }
#pragma unroll
            for (int t = 0; t < C::FN; t++) {
                const int nl = wn * C::TN + t * 8 + r, kl = kk * 4 + c;
                bf[t] = TB ? sB[kl * (C::BN + PAD) + nl] : sB[nl * (BK + PAD) + kl];
            }
#pragma unroll
            for (int s = 0; s < C::FM; s++)
#pragma unroll
                for (int t = 0; t < C::FN; t++) mma884(acc[s][t][0], acc[s][t][1], af[s], bf[t]);
        }
    }
    cp_async_wait<0>();
    __syncthreads();
}

}  // namespace dmma
}  // namespace bsrg
