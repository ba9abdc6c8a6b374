// bsrg_ctx: stream, solver handles and a growable device workspace.
#pragma once
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <vector>

#include "bsrg_internal.h"

struct bsrg_stage_event {
    int stage;
    cudaEvent_t start, stop;
};

// R^k tables of one basis for k = 0..kmax, resident in the assembly's
// zero-margined layout (built once, shared by every partial wave of the basis)
struct bsrg_tables {
    const bsrg_basis *basis;
    int kmax;
    double *rkbp;            // (kmax+1) consecutive tables
    size_t table_doubles;    // doubles per multipole
};

struct bsrg_ctx {
    int device;
    cudaStream_t stream;
    cublasHandle_t blas;
    cusolverDnHandle_t solver;
    void *ws;                 // device workspace
    size_t ws_bytes;
    void *pinned;             // pinned host staging buffer
    size_t pinned_bytes;
    cudaEvent_t ev_stage;     // guards reuse of the pinned buffer
    // stage timing (off unless bsrg_ctx_set_timing)
    int timing;
    std::vector<bsrg_stage_event> *events;   // recorded, not yet read
    std::vector<cudaEvent_t> *pool;          // free events
    double stage_ms[BSRG_NSTAGE];
    int stage_launches[BSRG_NSTAGE];
    double stage_flops[BSRG_NSTAGE];        // executed flops (counted where the library knows them)
    const bsrg_tables *tables;               // resident tables to use, or NULL
    std::vector<int> *last_ipsol;            // channel solution offsets of the last diag_hd
    void *pw_buf;                            // device buffers of bsrg_partial_wave_solve (kept between calls)
    size_t pw_bytes;
    bsrg_basis *pw_basis;                    // basis of the last bsrg_partial_wave_solve, reused while
    std::vector<double> *pw_knots;           //   ks and the knots are unchanged
    int pw_ks;
    int refine;                              // FP64 refinement of the eigenpairs in diag_hd (default on)
    int precision;                           // 0 FP64 (default), 1 mixed (tensor-core assembly contraction)
    int eig_mode;                            // dense eigensolver of diag_hd: 0 by size, 1 library's, 2 cuSOLVER's
    double *rf_buf;                          // per-pair correction | residual of the last refined diag_hd
    size_t rf_cap;                           //   (doubles held)
    int rf_n;                                //   (pairs recorded)
    int chan_fallbacks;                      // channel solves redone on the library path (orthogonality check)
    cudaStream_t aux_stream;                 // high-priority second stream (the band reduction's panels), or 0
    cudaEvent_t aux_ev[2];                   //   its hand-off events
};

namespace bsrg {

// carve aligned sub-buffers out of one allocation
struct Arena {
    char *base;
    size_t off, cap;
    template <class T> T *take(size_t n)
    {
        off = (off + 255) & ~(size_t)255;
        T *p = (T *)(base + off);
        off += n * sizeof(T);
        return p;
    }
};

// make sure the context workspace holds at least `bytes`; synchronises the
// stream before replacing a smaller buffer.
int ctx_reserve(bsrg_ctx *c, size_t bytes);
int ctx_reserve_pinned(bsrg_ctx *c, size_t bytes);

// stage timing helpers: no-ops unless timing is on
void stage_begin(bsrg_ctx *c, int stage);
void stage_end(bsrg_ctx *c, int stage, int launches = 1);
int stage_collect(bsrg_ctx *c);   // waits for recorded events and accumulates

// tridiagonal divide and conquer (tridiag_dc.cu)
size_t dc_workspace_bytes(int n);
size_t dc_pinned_bytes(int n);
int tridiag_dc(cudaStream_t st, int n, double *d, const double *e, double *w, double *Z, long ldz, void *ws_base,
               size_t ws_bytes, void *pinned, size_t pinned_bytes, double *gemm_flops, int *launches);

// two-stage dense symmetric eigensolver (syevd2.cu)
size_t syevd2_workspace_doubles(int n);
int dense_syevd(bsrg_ctx *c, int n, const double *A, long lda, double *w, double *Z, long ldz, double *ws,
                size_t ws_doubles, void *pinned, size_t pinned_bytes, int *launches);

// the channel eigenproblems of diag_hd (chan_eig.cu)
bool chan_own_ok(int ns, int ks, int npad, int device);
size_t chan_own_workspace_doubles(int nch, int npad, int ks);
int chan_own_solve(bsrg_ctx *c, const bsrg_basis *b, const double *hcc, int nch, int npad, const int *d_s0,
                   const int *d_nsol, double *AA, double *Wv, int *d_info, double *ws, int *d_flag);

// dense Cholesky and triangular solves (dense_chol.cu)
size_t chol_workspace_doubles(int n);
int dpotrf_lower(int n, double *C, long ldc, double *Linv, double *tmp, int *info, cudaStream_t s, int *launches);
int trsm_lower_left(int n, int m, const double *L, long ldl, const double *Linv, double *B, long ldb, bool trans,
                    double *tmp, size_t tmp_doubles, cudaStream_t s, int *launches);
int sygst_lower(int n, double *A, long lda, const double *L, long ldl, const double *Linv, double *T, double *tmp,
                size_t tmp_doubles, cudaStream_t s, int *launches);
int mirror_lower(int n, double *A, long lda, cudaStream_t s);

// eigenpair refinement (refine.cu)
size_t refine_workspace_doubles(int n);
int refine_prepare(int n, const double *A, long lda, double *F, cudaStream_t s);
int refine_apply(int n, const double *F, double *V, long ldv, double *lam, double *work, double *corr, double *resid,
                 int *flag, cudaStream_t s, void *oz_ws = nullptr, size_t oz_bytes = 0, int *oz_err = nullptr);

}  // namespace bsrg
