// FP64 residual refinement of symmetric eigenpairs (no counterpart in the
// reference, whose DSYEV result is used as is).
//
// For each eigenpair (lambda_j, v_j) of the khm x khm matrix A that diag_hd
// diagonalises (diag_hd.f90:312), the residual r_j = A v_j - lambda_j v_j is
// formed in FP64 and the Rayleigh quotient replaces the eigenvalue:
//     lambda_j <- lambda_j + v_j^T r_j / v_j^T v_j,
// whose error is ~ ||r_j||^2 / gap_j plus the rounding of v^T r, which scales
// with |v_j|^T |A| |v_j| instead of ||A||.  Raw FP64 eigensolvers (LAPACK DSYEV
// and GPU solvers alike) leave every eigenvalue with an error ~eps ||A||; here
// ||A|| ~ 1e7 (kinetic energies of the 1e-3 a.u. first knot interval) while the
// physical eigenvalues are O(1), so the correction is what makes eigenvalues
// agree per eigenvalue, not only relative to the spectral radius.
//
// A V is one FP64 tensor-core GEMM (dmma.cuh) whose epilogue reduces, per
// column j and 128-row tile, sum v (AV - lambda v), sum (AV - lambda v)^2 and
// sum v^2; the partial sums are added in a fixed order afterwards, so the
// result is bitwise repeatable and A V is never written to memory.
#include "ctx.h"
#include "dgemm.h"
#include "dmma.cuh"

namespace bsrg {

// F(i,j) = F(j,i) = A(i,j) for i >= j (the lower triangle of A, lda) -- 32x32 tiles
__global__ void symmetrize_lower_kernel(int n, const double *__restrict__ A, long lda, double *__restrict__ F,
                                        long ldf)
{
    __shared__ double tile[32][33];
    const int bi = blockIdx.x, bj = blockIdx.y;   // tile row, tile column
    if (bi < bj) return;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int q = ty; q < 32; q += 8) {
        const int i = bi * 32 + tx, j = bj * 32 + q;
        double v = 0.0;
        if (i < n && j < n && i >= j) v = A[i + (long)lda * j];
        else if (i < n && j < n) v = A[j + (long)lda * i];   // diagonal tile, upper part: mirror
        tile[q][tx] = v;
        if (i < n && j < n) F[i + (long)ldf * j] = v;
    }
    __syncthreads();
    if (bi == bj) return;
    for (int q = ty; q < 32; q += 8) {
        const int i = bj * 32 + tx, j = bi * 32 + q;     // F(bj-tile rows, bi-tile cols) = tile^T
        if (i < n && j < n) F[i + (long)ldf * j] = tile[tx][q];
    }
}

// partial sums of the Rayleigh correction: P[(tm*3 + w)*n + j], w = 0: sum v r,
// 1: sum r^2, 2: sum v^2 over rows of M tile tm (r = (F V)(i,j) - lambda_j V(i,j))
__global__ void __launch_bounds__(dmma::Sq::NT) refine_gemm_kernel(int n, const double *__restrict__ F, long ldf,
                                                               const double *__restrict__ V, long ldv,
                                                               const double *__restrict__ lam, double *__restrict__ P)
{
    extern __shared__ __align__(16) double smem[];
    using C = dmma::Sq;
    const int m0 = blockIdx.x * C::BM, n0 = blockIdx.y * C::BN;
    double acc[C::FM][C::FN][2];
    dmma::tile_mma<C, false, false>(acc, smem, F, ldf, V, ldv, n, n, 0, n, m0, n0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm = warp & 1, wn = warp >> 1, r = lane >> 2, q = lane & 3;
    double *red = smem;   // [2 wm][128 columns][3] after the pipeline has drained
#pragma unroll
    for (int t = 0; t < 4; t++)
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int cl = wn * 32 + t * 8 + 2 * q + j, col = n0 + cl;
            double svr = 0.0, srr = 0.0, svv = 0.0;
            if (col < n) {
                const double lj = lam[col];
#pragma unroll
                for (int s = 0; s < 8; s++) {
                    const int row = m0 + wm * 64 + s * 8 + r;
                    if (row < n) {
                        const double v = V[row + (long)ldv * col];
                        const double res = acc[s][t][j] - lj * v;
                        svr += v * res;
                        srr += res * res;
                        svv += v * v;
                    }
                }
            }
#pragma unroll
            for (int o = 4; o < 32; o <<= 1) {
                svr += __shfl_xor_sync(0xffffffffu, svr, o);
                srr += __shfl_xor_sync(0xffffffffu, srr, o);
                svv += __shfl_xor_sync(0xffffffffu, svv, o);
            }
            if (r == 0) {
                red[(wm * 128 + cl) * 3 + 0] = svr;
                red[(wm * 128 + cl) * 3 + 1] = srr;
                red[(wm * 128 + cl) * 3 + 2] = svv;
            }
        }
    __syncthreads();
    for (int idx = threadIdx.x; idx < 128 * 3; idx += C::NT) {
        const int cl = idx / 3, w = idx % 3, col = n0 + cl;
        if (col < n) P[((long)blockIdx.x * 3 + w) * n + col] = red[cl * 3 + w] + red[(128 + cl) * 3 + w];
    }
}

// lambda_j += sum v r / sum v^2 (tiles added in order); resid_j = ||r_j||, corr_j = the correction
__global__ void refine_finalize_kernel(int n, int ntm, const double *__restrict__ P, double *lam, double *corr,
                                       double *resid)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double vr = 0.0, rr = 0.0, vv = 0.0;
    for (int tm = 0; tm < ntm; tm++) {
        vr += P[((long)tm * 3 + 0) * n + j];
        rr += P[((long)tm * 3 + 1) * n + j];
        vv += P[((long)tm * 3 + 2) * n + j];
    }
    const double c = vv > 0.0 ? vr / vv : 0.0;
    lam[j] += c;
    if (corr) corr[j] = c;
    if (resid) resid[j] = vv > 0.0 ? sqrt(rr / vv) : 0.0;
}

// Keep the eigenvalues ascending (DSYEV's order): corrections are ~eps ||A||, so
// only eigenvalues closer than that can change places.  Odd-even passes over
// adjacent pairs swap the values, the vectors' columns and the per-pair data;
// one CTA, at most `max_pass` passes (each pass moves an element by one place).
__global__ void refine_order_kernel(int n, double *lam, double *V, long ldv, double *corr, double *resid,
                                    int max_pass, int *unsorted)
{
    __shared__ int swapped;
    __shared__ int list[1024];
    __shared__ int nl;
    for (int pass = 0; pass < max_pass; pass++) {
        if (threadIdx.x == 0) { swapped = 0; nl = 0; }
        __syncthreads();
        const int par = pass & 1;
        for (int i = 2 * threadIdx.x + par; i + 1 < n; i += 2 * blockDim.x)
            if (lam[i] > lam[i + 1]) {
                const int s = atomicAdd(&nl, 1);
                if (s < 1024) list[s] = i;
                swapped = 1;
            }
        __syncthreads();
        const int cnt = nl < 1024 ? nl : 1024;
        for (int q = 0; q < cnt; q++) {
            const int i = list[q];
            for (int r = threadIdx.x; r < n; r += blockDim.x) {
                double *a = V + (long)ldv * i + r, *b = V + (long)ldv * (i + 1) + r;
                const double t = *a;
                *a = *b;
                *b = t;
            }
            if (threadIdx.x == 0) {
                double t = lam[i]; lam[i] = lam[i + 1]; lam[i + 1] = t;
                if (corr) { t = corr[i]; corr[i] = corr[i + 1]; corr[i + 1] = t; }
                if (resid) { t = resid[i]; resid[i] = resid[i + 1]; resid[i + 1] = t; }
            }
        }
        __syncthreads();
        const int any = swapped;
        __syncthreads();
        if (!any) {
            if (threadIdx.x == 0) *unsorted = 0;
            return;
        }
    }
    if (threadIdx.x == 0) *unsorted = 1;
}

size_t refine_workspace_doubles(int n)
{
    const size_t ntm = (size_t)(n + dmma::Sq::BM - 1) / dmma::Sq::BM;
    return (size_t)n * n + ntm * 3 * n + 64;
}

int symmetrize_lower(int n, const double *A, long lda, double *F, long ldf, cudaStream_t s)
{
    dim3 g((unsigned)((n + 31) / 32), (unsigned)((n + 31) / 32)), blk(32, 8);
    symmetrize_lower_kernel<<<g, blk, 0, s>>>(n, A, lda, F, ldf);
    return cuda_fail(cudaGetLastError(), "symmetrize");
}

// F (n*n doubles of workspace) <- the lower triangle of A mirrored: call before
// the eigensolver overwrites A.
int refine_prepare(int n, const double *A, long lda, double *F, cudaStream_t s)
{
    dim3 g((unsigned)((n + 31) / 32), (unsigned)((n + 31) / 32)), blk(32, 8);
    symmetrize_lower_kernel<<<g, blk, 0, s>>>(n, A, lda, F, n);
    return cuda_fail(cudaGetLastError(), "refine: symmetrize");
}

// After the eigensolver: lam (n) refined in place, V (ldv) reordered if needed;
// corr/resid (n, device) may be NULL.  P needs ntm*3*n doubles; flag one int.
int refine_apply(int n, const double *F, double *V, long ldv, double *lam, double *P, double *corr, double *resid,
                 int *flag, cudaStream_t s)
{
    constexpr int bytes = dmma::Smem<dmma::Sq, false, false>::BYTES;
    static_assert(bytes >= 2 * 128 * 3 * 8, "epilogue reduction fits the pipeline's shared memory");
    cudaError_t e = cudaFuncSetAttribute(refine_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "refine: shared memory attribute");
    const int ntm = (n + dmma::Sq::BM - 1) / dmma::Sq::BM;
    dim3 g((unsigned)ntm, (unsigned)((n + dmma::Sq::BN - 1) / dmma::Sq::BN));
    refine_gemm_kernel<<<g, dmma::Sq::NT, bytes, s>>>(n, F, n, V, ldv, lam, P);
    refine_finalize_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, ntm, P, lam, corr, resid);
    refine_order_kernel<<<1, 1024, 0, s>>>(n, lam, V, ldv, corr, resid, 64, flag);
    return cuda_fail(cudaGetLastError(), "refine launch");
}

}  // namespace bsrg
