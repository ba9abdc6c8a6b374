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
// A V is one FP64 tensor-core GEMM (dmma.cuh) whose epilogue writes the
// residuals R = A V - V diag(lambda) and reduces, per column j and 128-row tile,
// sum r^2 (the residual norms); the partial sums are added in a fixed order, so
// the result is bitwise repeatable.
//
// The quotient's error ||r_j||^2 / gap_j is large where eigenvalues cluster (gaps
// of 1e-3 among O(1) eigenvalues of a matrix of norm 1e8: the two members of a
// close pair move apart or together by 1e-11 and more).  So the quotient is
// taken one step further, to a Rayleigh-Ritz value: for every j the window of
// pairs [j - 8, j + 8] gives the symmetric matrix M(k, l) = v_k^T A v_l
// = v_k^T r_l + lambda_l v_k^T v_l (from the banded products of V with R and
// with itself, scaled by the vectors' norms), cyclic Jacobi rotations
// diagonalise it, and lambda_j becomes its Ritz value in j's place of the
// window.  The diagonal of M is the Rayleigh quotient; the rotations remove
// what the pairs inside the window contribute to one another's quotients.
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
// 1: sum r^2, 2: sum v^2 over rows of M tile tm (r = (F V)(i,j) - lambda_j V(i,j));
// r itself goes to R (n x n, leading dimension n)
__global__ void __launch_bounds__(dmma::Sq::NT) refine_gemm_kernel(int n, const double *__restrict__ F, long ldf,
                                                               const double *__restrict__ V, long ldv,
                                                               const double *__restrict__ lam, double *__restrict__ P,
                                                               double *__restrict__ R)
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
                        R[row + (long)n * col] = res;
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

// The residual epilogue of the mixed-precision form, whose A V comes from the digit product
// (tc_ozaki.cu) in R: R(i,j) -= lambda_j V(i,j) and the same per-tile partial sums as
// refine_gemm_kernel, P[(tm*3 + w)*n + j] over rows of 128-row tile tm.  One warp per column
// and tile (lanes over rows, shuffles in a fixed order), eight columns per CTA.
__global__ void __launch_bounds__(256) refine_resid_kernel(int n, const double *__restrict__ V, long ldv,
                                                           const double *__restrict__ lam, double *__restrict__ P,
                                                           double *__restrict__ R)
{
    const int lane = threadIdx.x & 31, col = blockIdx.y * 8 + (threadIdx.x >> 5), tm = blockIdx.x;
    if (col >= n) return;
    const double lj = lam[col];
    double svr = 0.0, srr = 0.0, svv = 0.0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int row = tm * 128 + q * 32 + lane;
        if (row < n) {
            const double v = V[row + (long)ldv * col];
            double *rp = R + row + (long)n * col;
            const double res = *rp - lj * v;
            *rp = res;
            svr += v * res;
            srr += res * res;
            svv += v * v;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        svr += __shfl_xor_sync(0xffffffffu, svr, o);
        srr += __shfl_xor_sync(0xffffffffu, srr, o);
        svv += __shfl_xor_sync(0xffffffffu, svv, o);
    }
    if (lane == 0) {
        P[((long)tm * 3 + 0) * n + col] = svr;
        P[((long)tm * 3 + 1) * n + col] = srr;
        P[((long)tm * 3 + 2) * n + col] = svv;
    }
}

// resid_j = ||r_j|| / ||v_j|| (tiles added in order)
__global__ void refine_finalize_kernel(int n, int ntm, const double *__restrict__ P, double *resid)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double vr = 0.0, rr = 0.0, vv = 0.0;
    for (int tm = 0; tm < ntm; tm++) {
        vr += P[((long)tm * 3 + 0) * n + j];
        rr += P[((long)tm * 3 + 1) * n + j];
        vv += P[((long)tm * 3 + 2) * n + j];
    }
    (void)vr;
    if (resid) resid[j] = vv > 0.0 ? sqrt(rr / vv) : 0.0;
}

constexpr int RR_HW = 8;                    // half-width of the Rayleigh-Ritz window
constexpr int RR_W = 2 * RR_HW + 1;         // pairs in a window
constexpr int RR_BW = 2 * RR_HW;            // half-width of the band of products a window needs
constexpr int RR_ND = 2 * RR_BW + 1;        // products per column

// Bd(j, d) = v_{j+d}^T r_j and Gd(j, d) = v_{j+d}^T v_j at [j RR_ND + d + RR_BW], |d| <= RR_BW (zero
// where j + d is outside 0..n-1); one CTA per 32 columns, rows through shared memory 32 at a time
__global__ void __launch_bounds__(256) refine_band_kernel(int n, const double *__restrict__ V, long ldv,
                                                          const double *__restrict__ R, double *__restrict__ Bd,
                                                          double *__restrict__ Gd)
{
    __shared__ double Vs[32][32 + 2 * RR_BW + 1];      // columns j0 - RR_BW .. j0 + 31 + RR_BW
    __shared__ double Rs[32][33];
    constexpr int NP = 32 * RR_ND, PT = (NP + 255) / 256;
    const int j0 = blockIdx.x * 32, tid = threadIdx.x;
    double ab[PT], ag[PT];
#pragma unroll
    for (int u = 0; u < PT; u++) ab[u] = ag[u] = 0.0;
    for (int r0 = 0; r0 < n; r0 += 32) {
        __syncthreads();
        for (int e = tid; e < 32 * (32 + 2 * RR_BW); e += 256) {
            const int rr = e & 31, c = e >> 5, col = j0 - RR_BW + c, row = r0 + rr;
            Vs[rr][c] = (row < n && col >= 0 && col < n) ? V[row + ldv * (long)col] : 0.0;
        }
        for (int e = tid; e < 32 * 32; e += 256) {
            const int rr = e & 31, c = e >> 5, col = j0 + c, row = r0 + rr;
            Rs[rr][c] = (row < n && col < n) ? R[row + (long)n * col] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < PT; u++) {
            const int p = tid + 256 * u;
            if (p < NP) {
                const int jl = p / RR_ND, d = p % RR_ND;     // column j0 + jl, partner j0 + jl + d - RR_BW
                double sb = 0.0, sg = 0.0;
#pragma unroll 8
                for (int rr = 0; rr < 32; rr++) {
                    const double vk = Vs[rr][jl + d];
                    sb = fma(vk, Rs[rr][jl], sb);
                    sg = fma(vk, Vs[rr][jl + RR_BW], sg);
                }
                ab[u] += sb;
                ag[u] += sg;
            }
        }
    }
#pragma unroll
    for (int u = 0; u < PT; u++) {
        const int p = tid + 256 * u;
        if (p < NP) {
            const int jl = p / RR_ND, d = p % RR_ND, j = j0 + jl;
            if (j < n) {
                Bd[(long)j * RR_ND + d] = ab[u];
                Gd[(long)j * RR_ND + d] = ag[u];
            }
        }
    }
}

// One warp per eigenvalue j: the window [lo, hi] = [j - RR_HW, j + RR_HW] cut to 0..n-1, its matrix
// M(k, l) = (v_k^T r_l + lambda_l v_k^T v_l) / (|v_k| |v_l|), symmetrised, diagonalised by cyclic
// Jacobi rotations (each zeroes one off-diagonal pair), and lamw_j = its (j - lo)-th smallest value.
__global__ void __launch_bounds__(256) refine_window_kernel(int n, const double *__restrict__ lam,
                                                            const double *__restrict__ Bd,
                                                            const double *__restrict__ Gd, double *__restrict__ lamw)
{
    __shared__ double S[8][RR_W][RR_W + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int j = blockIdx.x * 8 + warp;
    if (j >= n) return;
    const int lo = max(0, j - RR_HW), hi = min(n - 1, j + RR_HW), w = hi - lo + 1;
    double (*A)[RR_W + 1] = S[warp];
    for (int e = lane; e < w * w; e += 32) {
        const int k = e / w, l = e % w, gk = lo + k, gl = lo + l;
        const double mkl = Bd[(long)gl * RR_ND + (gk - gl + RR_BW)] + lam[gl] * Gd[(long)gl * RR_ND + (gk - gl + RR_BW)];
        const double mlk = Bd[(long)gk * RR_ND + (gl - gk + RR_BW)] + lam[gk] * Gd[(long)gk * RR_ND + (gl - gk + RR_BW)];
        const double nn = Gd[(long)gk * RR_ND + RR_BW] * Gd[(long)gl * RR_ND + RR_BW];
        A[k][l] = nn > 0.0 ? 0.5 * (mkl + mlk) / sqrt(nn) : (k == l ? lam[gk] : 0.0);
    }
    __syncwarp();
    for (int sweep = 0; sweep < 10; sweep++) {
        bool rotated = false;
        for (int p = 0; p < w - 1; p++)
            for (int q = p + 1; q < w; q++) {
                const double apq = A[p][q], app = A[p][p], aqq = A[q][q];
                if (!(fabs(apq) > 1e-19 * (fabs(app) + fabs(aqq))) || fabs(apq) < 1e-300) continue;
                rotated = true;
                // the rotation that zeroes (p, q): t = tan of its angle, the smaller root of
                // t^2 + 2 theta t - 1 = 0 with theta = (aqq - app) / (2 apq)
                const double th = (aqq - app) / (2.0 * apq);
                const double t = fabs(th) > 1e150 ? 0.5 / th : copysign(1.0, th) / (fabs(th) + sqrt(1.0 + th * th));
                const double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
                const bool mine = lane < w && lane != p && lane != q;
                double akp = 0.0, akq = 0.0;
                if (mine) { akp = A[lane][p]; akq = A[lane][q]; }
                __syncwarp();
                if (mine) {
                    const double np = c * akp - s * akq, nq = s * akp + c * akq;
                    A[lane][p] = np; A[p][lane] = np;
                    A[lane][q] = nq; A[q][lane] = nq;
                }
                if (lane == 0) {
                    A[p][p] = app - t * apq;
                    A[q][q] = aqq + t * apq;
                    A[p][q] = 0.0;
                    A[q][p] = 0.0;
                }
                __syncwarp();
            }
        if (!rotated) break;
    }
    const double dk = lane < w ? A[lane][lane] : 0.0;
    int rank = 0;
    for (int m = 0; m < w; m++) {
        const double dm = A[m][m];
        rank += (dm < dk || (dm == dk && m < lane)) ? 1 : 0;
    }
    if (lane < w && rank == j - lo) lamw[j] = dk;
}

// corr_j = lamw_j - lambda_j, lambda_j = lamw_j
__global__ void refine_commit_kernel(int n, const double *__restrict__ lamw, double *lam, double *corr)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    if (corr) corr[j] = lamw[j] - lam[j];
    lam[j] = lamw[j];
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

// refine_apply's work: tile sums (ntm 3 n), R (n n), the banded products (2 RR_ND n), the Ritz values (n)
static size_t refine_work_doubles(int n)
{
    const size_t ntm = (size_t)(n + dmma::Sq::BM - 1) / dmma::Sq::BM;
    return ntm * 3 * n + (size_t)n * n + (2 * RR_ND + 1) * (size_t)n + 64;
}

size_t refine_workspace_doubles(int n) { return (size_t)n * n + refine_work_doubles(n); }

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
// corr/resid (n, device) may be NULL.  work: refine_work_doubles(n); flag one int.
// oz_ws (ozaki_ws_bytes(n, n, n, 8) bytes) selects the mixed-precision form's A V
// (digit product, wait and input errors in *oz_err); NULL the FP64 tensor-core GEMM.
int refine_apply(int n, const double *F, double *V, long ldv, double *lam, double *work, double *corr, double *resid,
                 int *flag, cudaStream_t s, void *oz_ws, size_t oz_bytes, int *oz_err)
{
    constexpr int bytes = dmma::Smem<dmma::Sq, false, false>::BYTES;
    static_assert(bytes >= 2 * 128 * 3 * 8, "epilogue reduction fits the pipeline's shared memory");
    cudaError_t e = smem_attr(refine_gemm_kernel, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "refine: shared memory attribute");
    const int ntm = (n + dmma::Sq::BM - 1) / dmma::Sq::BM;
    dim3 g((unsigned)ntm, (unsigned)((n + dmma::Sq::BN - 1) / dmma::Sq::BN));
    double *P = work, *R = P + (size_t)ntm * 3 * n, *Bd = R + (size_t)n * n, *Gd = Bd + (size_t)RR_ND * n;
    double *lamw = Gd + (size_t)RR_ND * n;
    if (oz_ws) {
        // mixed-precision form: A V from 8-bit digits on the tensor cores, then the residual epilogue
        static_assert(dmma::Sq::BM == 128, "the residual epilogue's tiles are the GEMM's");
        int rc = ozaki_gemm(n, n, n, 1.0, F, n, V, ldv, 0.0, R, n, 8, oz_ws, oz_bytes, oz_err, s);
        if (rc != BSRG_OK) return rc;
        refine_resid_kernel<<<dim3((unsigned)ntm, (unsigned)((n + 7) / 8)), 256, 0, s>>>(n, V, ldv, lam, P, R);
    } else {
        refine_gemm_kernel<<<g, dmma::Sq::NT, bytes, s>>>(n, F, n, V, ldv, lam, P, R);
    }
    refine_finalize_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, ntm, P, resid);
    refine_band_kernel<<<(n + 31) / 32, 256, 0, s>>>(n, V, ldv, R, Bd, Gd);
    refine_window_kernel<<<(n + 7) / 8, 256, 0, s>>>(n, lam, Bd, Gd, lamw);
    refine_commit_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, lamw, lam, corr);
    refine_order_kernel<<<1, 1024, 0, s>>>(n, lam, V, ldv, corr, resid, 64, flag);
    return cuda_fail(cudaGetLastError(), "refine launch");
}

}  // namespace bsrg
