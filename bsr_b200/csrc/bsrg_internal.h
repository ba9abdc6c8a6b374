// Internal declarations shared by the bsrgpu translation units.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <string>

#include "../../include/bsr_b200.h"

#define BSRG_MAXKS 16

// Device-resident B-spline basis (spline_param + spline_grid + spline_galerkin
// module state of the reference, libs/BS/spline_*.f90).  All arrays keep the
// Fortran column-major layout, 0-based:
//   t[ns+ks]; gr/grm/grw (nv,ks) at [iv + nv*m];
//   bsp/bsq (nv+1,ks,ks) at [iv + (nv+1)*(m + ks*ith)], bspd adds index d (0,1);
//   band matrices (ns,ks) at [i + ns*jcol] (lower-column storage).
struct bsrg_basis {
    int ks, ns, nv, ml, me;
    double h;
    double gx[BSRG_MAXKS], gw[BSRG_MAXKS];    // host copies of the Gauss rule
    double *t, *gr, *grm, *grw, *bsp, *bsq, *bspd;
    double *sb, *r1, *rm1, *rm2, *rm3, *db1, *db2;
    int device;
};

namespace bsrg {

void set_error(const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *where);

// Raises a kernel's dynamic shared-memory limit to `bytes` on the current device and never lowers
// it: threads that launch the same kernel with different sizes on their own streams cannot undo
// one another's limit between setting it and launching.
cudaError_t smem_attr_raw(const void *func, int bytes);
template <typename F> inline cudaError_t smem_attr(F *func, size_t bytes)
{
    return smem_attr_raw((const void *)func, (int)bytes);
}

inline int ik_of(int ks) { return ks * (ks + 1) / 2; }

// Gauss-Legendre nodes/weights on [0,1], ascending (Newton on P_k).
void gauss_legendre(int k, double *x, double *w);

// kernels launched by the C-ABI layer
int launch_basis_tables(bsrg_basis *b, cudaStream_t s);
int launch_mrm(const bsrg_basis *b, int mm, double *rm, cudaStream_t s);
int launch_rk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd, cudaStream_t s);
int launch_mrk_cell(const bsrg_basis *b, const double *rkd1, const double *rkd2, const double *rkd,
                    double *rkb, int ldp, cudaStream_t s);
int launch_nkmk_moments(const bsrg_basis *b, int k, int sym, double *rkd1, double *rkd2, double *rkd,
                        cudaStream_t s);
int launch_mrk_cell_scaled(const bsrg_basis *b, const double *rkd1, const double *rkd2, const double *rkd,
                           double fine, double *rkb, int ldp, cudaStream_t s);
int launch_mnk_cell(const bsrg_basis *b, const double *rkd1, const double *rkd2, const double *rkd, double fine,
                    double *rkb, int ldp, cudaStream_t s);
int launch_tk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd, cudaStream_t s);
int launch_mtk_cell(const bsrg_basis *b, int k, const double *rkd1, const double *rkd2, const double *rkd,
                    double fine, double *rkb, int ldp, cudaStream_t s);
int launch_vw_moments(const bsrg_basis *b, int k, int mode, double *rkd1, double *rkd2, double *rkd3, double *rkd4,
                      double *rkd, double *tmp, cudaStream_t s);
int launch_mvk_cell(const bsrg_basis *b, const double *rkd1, const double *rkd2, const double *rkd3,
                    const double *rkd4, const double *rkd, double fine, double *rkb, int ldp, cudaStream_t s);
int launch_mqk_cell(const bsrg_basis *b, const double *rkd1, const double *rkd2, const double *rkd3,
                    const double *rkd4, const double *rkd, double fine, double *rkb, int ldp, cudaStream_t s);
int launch_density(int ns, int ks, double *d, const double *p1, const double *p2, char type, cudaStream_t s);
int launch_convol(int ns, int ks, double *a, const double *d, const double *rkb, int ldp, int icase,
                  char si, char sj, cudaStream_t s);
int launch_sum_amb(int ns, int ks, const double *a, const double *b, char sym, double *out, cudaStream_t s);
int tf32x3_gemm(int m, int n, int k, double alpha, const double *A, long lda, const double *B, long ldb, double beta,
                double *C, long ldc, int *err, cudaStream_t s);
size_t ozaki_ws_bytes(int m, int n, int k, int slices);
int ozaki_gemm(int m, int n, int k, double alpha, const double *A, long lda, const double *B, long ldb, double beta,
               double *C, long ldc, int slices, void *ws, size_t ws_bytes, int *err, cudaStream_t s);
int launch_bav(int ns, int ks, const double *b, const double *v, double *y, char type, char side, cudaStream_t s);
int launch_bvmv(int n, int k, const double *ar, char type, const double *x, const double *y, double *out,
                cudaStream_t s);

}  // namespace bsrg
