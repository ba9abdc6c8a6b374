// Batched FP64 GEMM on the DMMA tensor pipe (dmma.cuh), C = alpha op(A) op(B) + beta C.
//
// Used by diag_hd's block transform (the hand loops of diag_hd.f90:188-219),
// the eigenpair refinement and the dense eigensolver.  Batches are uniform in
// size; item b reads A + b*sA (or Ap[b] when a pointer array is given), and
// likewise for B and C.
#include "ctx.h"
#include "dgemm.h"
#include "dmma.cuh"

namespace bsrg {

template <bool TA, bool TB>
__global__ void __launch_bounds__(dmma::NT) dgemm_kernel(DgemmBatch p)
{
    extern __shared__ __align__(16) double smem[];
    const int b = blockIdx.z;
    const double *A = p.Ap ? p.Ap[b] : p.A + (long)b * p.sA;
    const double *B = p.Bp ? p.Bp[b] : p.B + (long)b * p.sB;
    double *C = p.Cp ? p.Cp[b] : p.C + (long)b * p.sC;
    const int m0 = blockIdx.x * dmma::BM, n0 = blockIdx.y * dmma::BN;
    double acc[8][4][2];
    dmma::tile_mma<TA, TB>(acc, smem, A, p.lda, B, p.ldb, p.m, p.n, p.k, m0, n0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm = warp & 1, wn = warp >> 1, r = lane >> 2, q = lane & 3;
#pragma unroll
    for (int s = 0; s < 8; s++) {
        const int row = m0 + wm * 64 + s * 8 + r;
        if (row >= p.m) continue;
#pragma unroll
        for (int t = 0; t < 4; t++)
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const int col = n0 + wn * 32 + t * 8 + 2 * q + j;
                if (col >= p.n) continue;
                double *cp = C + row + (long)col * p.ldc;
                double v = p.alpha * acc[s][t][j];
                if (p.beta != 0.0) v += p.beta * *cp;
                *cp = v;
            }
    }
}

template <bool TA, bool TB> static int launch(const DgemmBatch &p, int batch, cudaStream_t s)
{
    constexpr int bytes = dmma::Smem<TA, TB>::BYTES;
    cudaError_t e = cudaFuncSetAttribute(dgemm_kernel<TA, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "dgemm: shared memory attribute");
    dim3 g((unsigned)((p.m + dmma::BM - 1) / dmma::BM), (unsigned)((p.n + dmma::BN - 1) / dmma::BN), (unsigned)batch);
    dgemm_kernel<TA, TB><<<g, dmma::NT, bytes, s>>>(p);
    return cuda_fail(cudaGetLastError(), "dgemm launch");
}

int dgemm_batched(bool ta, bool tb, const DgemmBatch &p, int batch, cudaStream_t s)
{
    if (p.m < 0 || p.n < 0 || p.k < 0 || batch < 0) {
        set_error("dgemm: negative size (m=%d n=%d k=%d batch=%d)", p.m, p.n, p.k, batch);
        return BSRG_ERR_ARG;
    }
    if (batch > 65535) { set_error("dgemm: batch %d above 65535", batch); return BSRG_ERR_ARG; }
    if (p.m == 0 || p.n == 0 || batch == 0) return BSRG_OK;
    if (p.lda < (ta ? p.k : p.m) || p.ldb < (tb ? p.n : p.k) || p.ldc < p.m || p.lda < 1 || p.ldb < 1) {
        set_error("dgemm: leading dimension too small (lda=%ld ldb=%ld ldc=%ld for m=%d n=%d k=%d)", p.lda, p.ldb,
                  p.ldc, p.m, p.n, p.k);
        return BSRG_ERR_ARG;
    }
    if (!ta && !tb) return launch<false, false>(p, batch, s);
    if (!ta && tb) return launch<false, true>(p, batch, s);
    if (ta && !tb) return launch<true, false>(p, batch, s);
    return launch<true, true>(p, batch, s);
}

int dgemm(bool ta, bool tb, int m, int n, int k, double alpha, const double *A, long lda, const double *B, long ldb,
          double beta, double *C, long ldc, cudaStream_t s)
{
    DgemmBatch p{};
    p.m = m; p.n = n; p.k = k;
    p.A = A; p.lda = lda; p.B = B; p.ldb = ldb; p.C = C; p.ldc = ldc;
    p.alpha = alpha; p.beta = beta;
    return dgemm_batched(ta, tb, p, 1, s);
}

}  // namespace bsrg

using namespace bsrg;

extern "C" int bsrg_dgemm(char transa, char transb, int m, int n, int k, double alpha, const double *A, long lda,
                          long strideA, const double *B, long ldb, long strideB, double beta, double *C, long ldc,
                          long strideC, int batch, void *stream)
{
    auto tr = [](char t) { return t == 'T' || t == 't'; };
    if (!(tr(transa) || transa == 'N' || transa == 'n') || !(tr(transb) || transb == 'N' || transb == 'n')) {
        set_error("dgemm: trans must be 'N' or 'T'");
        return BSRG_ERR_ARG;
    }
    if ((!C || ((!A || !B) && k > 0)) && m > 0 && n > 0 && batch > 0) {
        set_error("dgemm: null matrix");
        return BSRG_ERR_ARG;
    }
    DgemmBatch p{};
    p.m = m; p.n = n; p.k = k;
    p.A = A; p.lda = lda; p.sA = strideA;
    p.B = B; p.ldb = ldb; p.sB = strideB;
    p.C = C; p.ldc = ldc; p.sC = strideC;
    p.alpha = alpha; p.beta = beta;
    return dgemm_batched(tr(transa), tr(transb), p, batch, (cudaStream_t)stream);
}
