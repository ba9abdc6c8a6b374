// Dense Cholesky factorisation and triangular solves for the generalized
// branch of diag_hd (an overlap with off-diagonal channel blocks).
//
// Reference: src/bsr/BSR_HD3/diag_hd.f90:268-284 (DPOTRF of the transformed
// overlap C, DSYGST(1,'L') of A) and :322-334 (DTRSM('Left','L','T') back-
// transformation of the eigenvectors), LAPACK_calls.f90.
//
// Blocked, right-looking, NB = 128:
//   chol_diag_kernel   factors one NB x NB diagonal block in shared memory
//                      (L_jj written in place) and writes its inverse L_jj^-1;
//   the panel          L_{>j,j} = C_{>j,j} L_jj^-T   one FP64 tensor-core GEMM;
//   the trailing block C_{>j,>j} -= L_{>j,j} L_{>j,j}^T   a GEMM over the tiles that
//                      reach its lower triangle.
// A triangular solve with many right-hand sides uses the stored inverses of the
// diagonal blocks: B_i <- L_ii^-1 B_i, then B_{>i} -= L_{>i,i} B_i (GEMMs), which
// keeps all the arithmetic on the tensor pipe.  DSYGST's A <- L^-1 A L^-T is
// two such solves with a transpose between them.
#include "ctx.h"
#include "dgemm.h"

namespace bsrg {

constexpr int CH_NB = 128;
constexpr int CH_LD = CH_NB + 1;

// factor the nb x nb diagonal block D (lower, ld) in place, write D^-1 (lower, ld CH_NB) to Dinv
__global__ void __launch_bounds__(256)
chol_diag_kernel(int nb, int j0, double *D, long ld, double *Dinv, int *info)
{
    extern __shared__ double cs[];
    double *S = cs;                          // [col][row], ld CH_LD
    double *x = S + (size_t)CH_NB * CH_LD;   // column temp
    const int tid = threadIdx.x;
    for (int q = tid; q < nb * nb; q += blockDim.x) {
        const int r = q % nb, c = q / nb;
        S[c * CH_LD + r] = r >= c ? D[r + ld * c] : 0.0;
    }
    __syncthreads();
    for (int k = 0; k < nb; k++) {
        if (tid == 0) {
            double d = S[k * CH_LD + k];
            if (!(d > 0.0)) {                // not positive definite: recorded, kept finite
                atomicCAS(info, 0, j0 + k + 1);
                d = 1.0;
            }
            S[k * CH_LD + k] = sqrt(d);
        }
        __syncthreads();
        const double dk = S[k * CH_LD + k];
        for (int i = k + 1 + tid; i < nb; i += blockDim.x) S[k * CH_LD + i] /= dk;
        __syncthreads();
        const int m = nb - k - 1;
        for (int q = tid; q < m * m; q += blockDim.x) {
            const int i = k + 1 + q % m, j = k + 1 + q / m;
            if (j <= i) S[j * CH_LD + i] -= S[k * CH_LD + i] * S[k * CH_LD + j];
        }
        __syncthreads();
    }
    for (int q = tid; q < nb * nb; q += blockDim.x) {
        const int r = q % nb, c = q / nb;
        if (r >= c) D[r + ld * c] = S[c * CH_LD + r];
    }
    // in-place inverse of the lower triangle, columns from the last (LAPACK dtrti2's order)
    for (int j = nb - 1; j >= 0; j--) {
        __syncthreads();
        if (tid == 0) S[j * CH_LD + j] = 1.0 / S[j * CH_LD + j];
        for (int i = j + 1 + tid; i < nb; i += blockDim.x) x[i] = S[j * CH_LD + i];
        __syncthreads();
        const double ajj = -S[j * CH_LD + j];
        // column j below the diagonal <- ajj * Tinv(j+1:, j+1:) x(j+1:)
        for (int i = j + 1 + tid; i < nb; i += blockDim.x) {
            double s = 0.0;
            for (int k = j + 1; k <= i; k++) s = fma(S[k * CH_LD + i], x[k], s);
            S[j * CH_LD + i] = ajj * s;
        }
    }
    __syncthreads();
    for (int q = tid; q < CH_NB * CH_NB; q += blockDim.x) {
        const int r = q % CH_NB, c = q / CH_NB;
        Dinv[q] = (r < nb && c < nb && r >= c) ? S[c * CH_LD + r] : 0.0;
    }
}

__global__ void copy2d_kernel(int m, int n, const double *__restrict__ src, long lds, double *dst, long ldd)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (size_t)m * n) return;
    const int r = (int)(q % m), c = (int)(q / m);
    dst[r + ldd * c] = src[r + lds * c];
}

// B (n x n) = A^T, 32 x 32 tiles
__global__ void transpose_kernel(int n, const double *__restrict__ A, long lda, double *B, long ldb)
{
    __shared__ double t[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int q = threadIdx.y; q < 32; q += blockDim.y) {
        const int r = bx + threadIdx.x, c = by + q;
        if (r < n && c < n) t[q][threadIdx.x] = A[r + lda * c];
    }
    __syncthreads();
    for (int q = threadIdx.y; q < 32; q += blockDim.y) {
        const int r = by + threadIdx.x, c = bx + q;
        if (r < n && c < n) B[r + ldb * c] = t[threadIdx.x][q];
    }
}

// A(i, j) = A(j, i) for i < j: the lower triangle mirrored into the upper, in place
__global__ void mirror_lower_kernel(int n, double *A, long lda)
{
    __shared__ double t[32][33];
    const int bi = blockIdx.x, bj = blockIdx.y;      // source tile rows bi, columns bj (lower: bi >= bj)
    if (bi < bj) return;
    for (int q = threadIdx.y; q < 32; q += blockDim.y) {
        const int r = bi * 32 + threadIdx.x, c = bj * 32 + q;
        t[q][threadIdx.x] = (r < n && c < n) ? A[r + lda * c] : 0.0;
    }
    __syncthreads();
    for (int q = threadIdx.y; q < 32; q += blockDim.y) {
        const int r = bj * 32 + threadIdx.x, c = bi * 32 + q;   // target (r, c) = source (c, r)
        if (r < n && c < n && r < c) A[r + lda * c] = t[threadIdx.x][q];
    }
}

int mirror_lower(int n, double *A, long lda, cudaStream_t s)
{
    dim3 g((unsigned)((n + 31) / 32), (unsigned)((n + 31) / 32));
    mirror_lower_kernel<<<g, dim3(32, 8), 0, s>>>(n, A, lda);
    return cuda_fail(cudaGetLastError(), "mirror_lower");
}

size_t chol_workspace_doubles(int n)
{
    const size_t nbk = (size_t)(n + CH_NB - 1) / CH_NB;
    return nbk * CH_NB * CH_NB + (size_t)n * CH_NB + 64;   // diagonal inverses | panel / solve temp
}

static int copy2d(int m, int n, const double *src, long lds, double *dst, long ldd, cudaStream_t s)
{
    const size_t cnt = (size_t)m * n;
    if (cnt == 0) return BSRG_OK;
    copy2d_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, s>>>(m, n, src, lds, dst, ldd);
    return cuda_fail(cudaGetLastError(), "copy2d");
}

// C = L L^T in place (lower); Linv receives the inverse of every diagonal block
// (CH_NB x CH_NB each), tmp n x CH_NB doubles; info (device) = first failing pivot (1-based)
int dpotrf_lower(int n, double *C, long ldc, double *Linv, double *tmp, int *info, cudaStream_t s, int *launches)
{
    const size_t smem = sizeof(double) * ((size_t)CH_NB * CH_LD + CH_NB);
    cudaError_t e = smem_attr(chol_diag_kernel, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "dpotrf: shared memory");
    int nl = 0;
    for (int j0 = 0, jb = 0; j0 < n; j0 += CH_NB, jb++) {
        const int nb = n - j0 < CH_NB ? n - j0 : CH_NB;
        double *D = C + j0 + ldc * j0, *Di = Linv + (size_t)jb * CH_NB * CH_NB;
        chol_diag_kernel<<<1, 256, smem, s>>>(nb, j0, D, ldc, Di, info);
        nl++;
        const int rem = n - j0 - nb;
        if (rem <= 0) continue;
        double *P = C + (j0 + nb) + ldc * j0;
        // panel: L_{>j,j} = C_{>j,j} (L_jj^-1)^T
        int rc = dgemm(false, true, rem, nb, nb, 1.0, P, ldc, Di, CH_NB, 0.0, tmp, rem, s);
        if (rc == BSRG_OK) rc = copy2d(rem, nb, tmp, rem, P, ldc, s);
        if (rc != BSRG_OK) return rc;
        // trailing: C_{>j,>j} -= L_{>j,j} L_{>j,j}^T, lower tiles only
        DgemmBatch g{};
        g.m = rem; g.n = rem; g.k = nb;
        g.A = P; g.lda = ldc; g.B = P; g.ldb = ldc;
        g.C = C + (j0 + nb) + ldc * (j0 + nb); g.ldc = ldc;
        g.alpha = -1.0; g.beta = 1.0; g.lowc = 1;
        rc = dgemm_batched(false, true, g, 1, s);
        if (rc != BSRG_OK) return rc;
        nl += 3;
    }
    if (launches) *launches += nl;
    return cuda_fail(cudaGetLastError(), "dpotrf");
}

// B (n x m) <- L^-1 B (trans = false) or L^-T B (trans = true), L from dpotrf_lower
int trsm_lower_left(int n, int m, const double *L, long ldl, const double *Linv, double *B, long ldb, bool trans,
                    double *tmp, size_t tmp_doubles, cudaStream_t s, int *launches)
{
    const int nbk = (n + CH_NB - 1) / CH_NB;
    // the diagonal-block products go through tmp in column chunks that fit it
    const int mc = (int)std::min<size_t>((size_t)m, tmp_doubles / CH_NB);
    if (mc < 1) { set_error("trsm: workspace too small"); return BSRG_ERR_NOMEM; }
    int nl = 0;
    for (int t = 0; t < nbk; t++) {
        const int ib = trans ? nbk - 1 - t : t;
        const int i0 = ib * CH_NB, nb = n - i0 < CH_NB ? n - i0 : CH_NB;
        const double *Di = Linv + (size_t)ib * CH_NB * CH_NB;
        double *Bi = B + i0;
        for (int c0 = 0; c0 < m; c0 += mc) {
            const int cn = m - c0 < mc ? m - c0 : mc;
            int rc = dgemm(trans, false, nb, cn, nb, 1.0, Di, CH_NB, Bi + ldb * c0, ldb, 0.0, tmp, nb, s);
            if (rc == BSRG_OK) rc = copy2d(nb, cn, tmp, nb, Bi + ldb * c0, ldb, s);
            if (rc != BSRG_OK) return rc;
            nl += 2;
        }
        int rc = BSRG_OK;
        if (!trans && i0 + nb < n) {
            // B_{>i} -= L_{>i,i} B_i
            const int rem = n - i0 - nb;
            rc = dgemm(false, false, rem, m, nb, -1.0, L + (i0 + nb) + ldl * i0, ldl, Bi, ldb, 1.0, B + i0 + nb, ldb, s);
            nl++;
        } else if (trans && i0 > 0) {
            // B_{<i} -= (L_{i,<i})^T B_i
            rc = dgemm(true, false, i0, m, nb, -1.0, L + i0, ldl, Bi, ldb, 1.0, B, ldb, s);
            nl++;
        }
        if (rc != BSRG_OK) return rc;
    }
    if (launches) *launches += nl;
    return BSRG_OK;
}

// A <- L^-1 A L^-T (DSYGST itype 1, lower): two left solves around a transpose; T is n x n scratch
int sygst_lower(int n, double *A, long lda, const double *L, long ldl, const double *Linv, double *T, double *tmp,
                size_t tmp_doubles, cudaStream_t s, int *launches)
{
    int rc = trsm_lower_left(n, n, L, ldl, Linv, A, lda, false, tmp, tmp_doubles, s, launches);
    if (rc != BSRG_OK) return rc;
    dim3 g((unsigned)((n + 31) / 32), (unsigned)((n + 31) / 32));
    transpose_kernel<<<g, dim3(32, 8), 0, s>>>(n, A, lda, T, n);
    if (launches) *launches += 1;
    rc = trsm_lower_left(n, n, L, ldl, Linv, T, n, false, tmp, tmp_doubles, s, launches);
    if (rc != BSRG_OK) return rc;
    return copy2d(n, n, T, n, A, lda, s);
}

}  // namespace bsrg
