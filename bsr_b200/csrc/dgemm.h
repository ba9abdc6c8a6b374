// Host interface of the FP64 DMMA GEMM (dgemm.cu).
#pragma once
#include <cuda_runtime.h>

namespace bsrg {

// A uniform batch: item b multiplies A + b*sA (or Ap[b]) by B + b*sB (or Bp[b])
// into C + b*sC (or Cp[b]); column-major, sizes of op(A) m x k, op(B) k x n.
struct DgemmBatch {
    int m, n, k;
    const double *A; long lda, sA;
    const double *B; long ldb, sB;
    double *C; long ldc, sC;
    const double *const *Ap;
    const double *const *Bp;
    double *const *Cp;
    double alpha, beta;
    int syma;          // op(A) = A square symmetric, only its lower triangle stored (no transpose)
    int lowc;          // compute only the tiles of C that reach the lower triangle (square C)
};

int dgemm_batched(bool ta, bool tb, const DgemmBatch &p, int batch, cudaStream_t s);
// with a workspace (work_doubles doubles), a single product with few tiles is split along K
int dgemm_ws(bool ta, bool tb, const DgemmBatch &p, int batch, cudaStream_t s, double *work, size_t work_doubles);
int dgemm(bool ta, bool tb, int m, int n, int k, double alpha, const double *A, long lda, const double *B, long ldb,
          double beta, double *C, long ldc, cudaStream_t s, double *work = nullptr, size_t work_doubles = 0);

}  // namespace bsrg
