// Batched FP64 GEMM on the DMMA tensor pipe (dmma.cuh), C = alpha op(A) op(B) + beta C.
//
// Used by diag_hd's block transform (the hand loops of diag_hd.f90:188-219),
// the eigenpair refinement and the dense eigensolver.  Batches are uniform in
// size; item b reads A + b*sA (or Ap[b] when a pointer array is given), and
// likewise for B and C.  The tile shape follows the output: 128 x 32 tiles
// when N <= 32, 32 x 128 when M <= 32, 128 x 128 otherwise.  With a workspace,
// a single product with too few tiles for the 148 SMs is split along K; the
// partial products are added in a fixed order, so results are repeatable.
#include <algorithm>

#include "ctx.h"
#include "dgemm.h"
#include "dmma.cuh"

namespace bsrg {

// S > 1: item b = blockIdx.z / S computes the K slice blockIdx.z % S into W
template <class C, bool TA, bool TB, bool SYMA = false>
__global__ void __launch_bounds__(C::NT) dgemm_kernel(DgemmBatch p, int S, int kchunk, double *W)
{
    extern __shared__ __align__(16) double smem[];
    if (p.lowc && (int)(blockIdx.y * C::BN) >= (int)(blockIdx.x + 1) * C::BM) return;   // wholly above the diagonal
    const int b = blockIdx.z / S, sp = blockIdx.z % S;
    const double *A = p.Ap ? p.Ap[b] : p.A + (long)b * p.sA;
    const double *B = p.Bp ? p.Bp[b] : p.B + (long)b * p.sB;
    double *Cm = p.Cp ? p.Cp[b] : p.C + (long)b * p.sC;
    const int m0 = blockIdx.x * C::BM, n0 = blockIdx.y * C::BN;
    const int kbeg = sp * kchunk, kend = min(p.k, kbeg + kchunk);
    double acc[C::FM][C::FN][2];
    dmma::tile_mma<C, TA, TB, SYMA>(acc, smem, A, p.lda, B, p.ldb, p.m, p.n, kbeg, kend, m0, n0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm = warp % C::WM, wn = warp / C::WM, r = lane >> 2, q = lane & 3;
    double *out = S > 1 ? W + (long)sp * p.m * p.n : Cm;
    const long ldo = S > 1 ? p.m : p.ldc;
    if (S == 1 && p.beta != 0.0) {
        // C is read here: every load of a row of tiles is issued before any is used, so the
        // epilogue waits for one memory latency per row of tiles instead of one per element
#pragma unroll
        for (int s = 0; s < C::FM; s++) {
            const int row = m0 + wm * C::TM + s * 8 + r;
            double old[C::FN][2];
#pragma unroll
            for (int t = 0; t < C::FN; t++)
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const int col = n0 + wn * C::TN + t * 8 + 2 * q + j;
                    old[t][j] = (row < p.m && col < p.n) ? out[row + (long)col * ldo] : 0.0;
                }
#pragma unroll
            for (int t = 0; t < C::FN; t++)
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const int col = n0 + wn * C::TN + t * 8 + 2 * q + j;
                    if (row < p.m && col < p.n) out[row + (long)col * ldo] = p.alpha * acc[s][t][j] + p.beta * old[t][j];
                }
        }
        return;
    }
#pragma unroll
    for (int s = 0; s < C::FM; s++) {
        const int row = m0 + wm * C::TM + s * 8 + r;
        if (row >= p.m) continue;
#pragma unroll
        for (int t = 0; t < C::FN; t++)
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const int col = n0 + wn * C::TN + t * 8 + 2 * q + j;
                if (col >= p.n) continue;
                double *cp = out + row + (long)col * ldo;
                *cp = S > 1 ? acc[s][t][j] : p.alpha * acc[s][t][j];
            }
    }
}

// C = alpha sum_s W_s + beta C (slices added in order)
__global__ void splitk_reduce_kernel(int m, int n, int S, const double *__restrict__ W, double alpha, double beta,
                                     double *C, long ldc)
{
    const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (idx >= (long)m * n) return;
    const int row = (int)(idx % m), col = (int)(idx / m);
    double s = 0.0;
    for (int q = 0; q < S; q++) s += W[(long)q * m * n + idx];
    double *cp = C + row + (long)col * ldc;
    double v = alpha * s;
    if (beta != 0.0) v += beta * *cp;
    *cp = v;
}

template <class C, bool TA, bool TB, bool SYMA = false>
static int launch(const DgemmBatch &p, int batch, int S, int kchunk, double *W, cudaStream_t s)
{
    constexpr int bytes = dmma::Smem<C, TA, TB>::BYTES;
    cudaError_t e = smem_attr(dgemm_kernel<C, TA, TB, SYMA>, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "dgemm: shared memory attribute");
    dim3 g((unsigned)((p.m + C::BM - 1) / C::BM), (unsigned)((p.n + C::BN - 1) / C::BN), (unsigned)(batch * S));
    dgemm_kernel<C, TA, TB, SYMA><<<g, C::NT, bytes, s>>>(p, S, kchunk, W);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "dgemm launch");
    if (S > 1) {
        const long mn = (long)p.m * p.n;
        splitk_reduce_kernel<<<(unsigned)((mn + 255) / 256), 256, 0, s>>>(p.m, p.n, S, W, p.alpha, p.beta, p.C,
                                                                          p.ldc);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "dgemm split-K reduce");
    }
    return BSRG_OK;
}

template <class C> static int launch_t(bool ta, bool tb, const DgemmBatch &p, int batch, int S, int kc, double *W,
                                       cudaStream_t s)
{
    if (!ta && !tb) return launch<C, false, false>(p, batch, S, kc, W, s);
    if (!ta && tb) return launch<C, false, true>(p, batch, S, kc, W, s);
    if (ta && !tb) return launch<C, true, false>(p, batch, S, kc, W, s);
    return launch<C, true, true>(p, batch, S, kc, W, s);
}

int dgemm_ws(bool ta, bool tb, const DgemmBatch &p, int batch, cudaStream_t s, double *work, size_t work_doubles)
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
    int bm = 128, bn = 128;
    if (p.n <= 32) bn = 32;
    else if (p.m <= 32) bm = 32;
    const long tiles = (long)((p.m + bm - 1) / bm) * ((p.n + bn - 1) / bn) * batch;
    int S = 1, kc = p.k;
    if (batch == 1 && work && tiles < 296 && p.k >= 512) {
        S = (int)std::min<long>({(296 + tiles - 1) / tiles, (long)p.k / 256, 16L});
        while (S > 1 && (size_t)S * p.m * p.n > work_doubles) S--;
        if (S > 1) {
            kc = ((p.k + S - 1) / S + dmma::BK - 1) / dmma::BK * dmma::BK;
            S = (p.k + kc - 1) / kc;
        }
    }
    if (S <= 1) { S = 1; kc = std::max(p.k, 1); }
    if (p.syma) {
        if (ta || p.m != p.k) { set_error("dgemm: a symmetric A must be square and not transposed"); return BSRG_ERR_ARG; }
        if (bn == 32) return tb ? launch<dmma::Tall, false, true, true>(p, batch, S, kc, work, s)
                                : launch<dmma::Tall, false, false, true>(p, batch, S, kc, work, s);
        return tb ? launch<dmma::Sq, false, true, true>(p, batch, S, kc, work, s)
                  : launch<dmma::Sq, false, false, true>(p, batch, S, kc, work, s);
    }
    if (p.lowc && p.m != p.n) { set_error("dgemm: lower-triangle output needs a square C"); return BSRG_ERR_ARG; }
    if (bn == 32) return launch_t<dmma::Tall>(ta, tb, p, batch, S, kc, work, s);
    if (bm == 32) return launch_t<dmma::Wide>(ta, tb, p, batch, S, kc, work, s);
    return launch_t<dmma::Sq>(ta, tb, p, batch, S, kc, work, s);
}

int dgemm_batched(bool ta, bool tb, const DgemmBatch &p, int batch, cudaStream_t s)
{
    return dgemm_ws(ta, tb, p, batch, s, nullptr, 0);
}

int dgemm(bool ta, bool tb, int m, int n, int k, double alpha, const double *A, long lda, const double *B, long ldb,
          double beta, double *C, long ldc, cudaStream_t s, double *work, size_t work_doubles)
{
    DgemmBatch p{};
    p.m = m; p.n = n; p.k = k;
    p.A = A; p.lda = lda; p.B = B; p.ldb = ldb; p.C = C; p.ldc = ldc;
    p.alpha = alpha; p.beta = beta;
    return dgemm_ws(ta, tb, p, 1, s, work, work_doubles);
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
